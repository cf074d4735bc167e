"""ctypes binding of oracle/_ref/liboracle.so, the plain-C restatement of the
hot path (cfd_oracle.c).  Test infrastructure: the checker for tests/,
__graft_entry__.smoke() and bench.py's CPU baseline when the reference build
is absent.  Same interface as refh.RefSolver.
"""
from __future__ import annotations

import ctypes as C
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "_ref" / "liboracle.so"
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_L = None


def available() -> bool:
    return PORT_LIB.exists()


def _lib():
    global _L
    if _L is None:
        if not PORT_LIB.exists():
            raise RuntimeError(f"{PORT_LIB} missing: run make -C {HERE} port")
        L = C.CDLL(str(PORT_LIB))
        L.oracle_connectivity.argtypes = [C.c_void_p, C.c_int, _ip, _ip]
        L.oracle_connectivity.restype = C.c_int64
        L.oracle_create.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]
        L.oracle_destroy.argtypes = [C.c_void_p]
        L.oracle_nnzb.argtypes = [C.c_void_p]
        L.oracle_nnzb.restype = C.c_int64
        L.oracle_structure.argtypes = [C.c_void_p, _ip, _ip]
        L.oracle_set_state.argtypes = [C.c_void_p, _dp, C.c_int64]
        L.oracle_get_state.argtypes = [C.c_void_p, _dp, C.c_int64]
        L.oracle_stages.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.oracle_jacobian.argtypes = [C.c_void_p, C.c_double, _dp, _dp]
        L.oracle_newton_step.argtypes = [C.c_void_p, C.c_double, _dp, C.POINTER(C.c_int)]
        L.oracle_nvars.argtypes = [C.c_void_p]
        L.oracle_nvars.restype = C.c_int
        L.oracle_sa_fields.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp]
        L.oracle_freeze_limiter.argtypes = [C.c_void_p, C.c_int]
        L.oracle_bsr_spmv.argtypes = [C.c_int, C.c_int, _ip, _ip, _dp, _dp, _dp, C.c_double, C.c_double]
        L.oracle_sgs_apply.argtypes = [C.c_int, C.c_int, _ip, _ip, _dp, _dp, _dp, C.c_int]
        L.oracle_bicgstab.argtypes = [C.c_int, C.c_int, _ip, _ip, _dp, C.c_int, C.c_double, C.c_double, C.c_int,
                                      _dp, _dp, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp, _dp]
        _L = L
    return _L


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def connectivity(mesh, kind: int):
    off = np.zeros(mesh.n_cells + 1, dtype=np.int32)
    cnt = _lib().oracle_connectivity(C.byref(mesh.view), kind, _i(off), None)
    val = np.zeros(max(cnt, 1), dtype=np.int32)
    _lib().oracle_connectivity(C.byref(mesh.view), kind, _i(off), _i(val))
    return off, val[:cnt]


class PortSolver:
    def __init__(self, mesh, cfg, bcs):
        self.n = mesh.n_cells
        self.nt = mesh.n_cells + mesh.n_faces - mesh.n_inner
        arr = (type(bcs[0]) * len(bcs))(*bcs)
        h = C.c_void_p()
        _lib().oracle_create(C.byref(mesh.view), C.byref(cfg), arr, len(bcs), C.byref(h))
        self._h = h
        self.nnzb = int(_lib().oracle_nnzb(self._h))
        self.nv = int(_lib().oracle_nvars(self._h))
        self.mesh = mesh  # the oracle keeps pointers into the mesh arrays

    def close(self):
        if getattr(self, "_h", None):
            _lib().oracle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def structure(self):
        rp = np.zeros(self.n + 1, dtype=np.int32)
        cols = np.zeros(self.nnzb, dtype=np.int32)
        _lib().oracle_structure(self._h, _i(rp), _i(cols))
        return rp, cols

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.nv, -1)
        _lib().oracle_set_state(self._h, _d(U), U.shape[1])

    def get_state(self):
        U = np.zeros((self.nv, self.n))
        _lib().oracle_get_state(self._h, _d(U), self.n)
        return U

    def stages(self):
        n, nt, nv = self.n, self.nt, self.nv
        q, grad, phi, res, lam = np.zeros(5 * nt), np.zeros(15 * nt), np.zeros(5 * n), np.zeros(nv * n), np.zeros(n)
        _lib().oracle_stages(self._h, _d(q), _d(grad), _d(phi), _d(res), _d(lam))
        out = {"q": q, "grad": grad, "phi": phi, "res": res, "lam": lam}
        if nv == 6:
            out.update(self.sa_fields())
        return out

    def sa_fields(self):
        """Spalart-Allmaras fields after the last residual: wall distance (n),
        nu_tilde (n), eddy viscosity (n_total), nu_tilde gradient (3 x n_total)."""
        n, nt = self.n, self.nt
        dist, nu, mut, gnu = np.zeros(n), np.zeros(n), np.zeros(nt), np.zeros(3 * nt)
        _lib().oracle_sa_fields(self._h, _d(dist), _d(nu), _d(mut), _d(gnu))
        return {"wall_dist": dist, "nu": nu, "mut": mut, "nu_grad": gnu}

    def freeze_limiter(self, frozen=True):
        """Keep the limiter values of the last evaluation (as the library's
        cfdg_solver_freeze_limiter)."""
        _lib().oracle_freeze_limiter(self._h, 1 if frozen else 0)

    def jacobian(self, cfl):
        alpha = np.zeros(self.n)
        vals = np.zeros(self.nnzb * self.nv * self.nv)
        _lib().oracle_jacobian(self._h, cfl, _d(alpha), _d(vals))
        return alpha, vals

    def newton_step(self, cfl):
        l2 = np.zeros(6)
        kr = (C.c_int * 2)()
        _lib().oracle_newton_step(self._h, cfl, _d(l2), kr)
        self.last_krylov = (kr[0], kr[1])
        return l2[:self.nv]


def bsr_spmv(row_ptr, cols, vals, bs, x, y=None, alpha=1.0, beta=0.0):
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros_like(x) if y is None else np.array(y, dtype=np.float64, copy=True)
    _lib().oracle_bsr_spmv(len(row_ptr) - 1, bs, _i(row_ptr), _i(cols), _d(vals), _d(x), _d(y), alpha, beta)
    return y


def sgs_apply(row_ptr, cols, vals, bs, r, sweeps=1):
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    r = np.ascontiguousarray(r, dtype=np.float64)
    z = np.zeros_like(r)
    _lib().oracle_sgs_apply(len(row_ptr) - 1, bs, _i(row_ptr), _i(cols), _d(vals), _d(r), _d(z), sweeps)
    return z


def bicgstab(row_ptr, cols, vals, bs, b, x0=None, precond=1, rel_tol=1e-8, abs_tol=1e-30, max_it=500):
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    it, st = C.c_int(), C.c_int()
    r0, rf = np.zeros(1), np.zeros(1)
    _lib().oracle_bicgstab(len(row_ptr) - 1, bs, _i(row_ptr), _i(cols), _d(vals), precond, rel_tol, abs_tol, max_it,
                           _d(x), _d(b), C.byref(it), C.byref(st), _d(r0), _d(rf))
    return x, {"iterations": it.value, "status": st.value, "initial": float(r0[0]), "final": float(rf[0])}


def newton_step(mesh, case, U0, cfl):
    """One oracle Newton step from U0: (L2 norms of R(U0), updated U)."""
    s = PortSolver(mesh, case.cfg, case.bcs)
    s.set_state(U0)
    l2 = s.newton_step(cfl)
    return l2, s.get_state()


def time_newton_steps(mesh, case, steps: int) -> float:
    """Seconds for `steps` oracle Newton iterations after one untimed one."""
    from cfd_b200.cases import freestream_state  # noqa: PLC0415
    s = PortSolver(mesh, case.cfg, case.bcs)
    s.set_state(freestream_state(case, mesh.n_cells))
    s.newton_step(case.cfg.cfl)
    t0 = time.perf_counter()
    for _ in range(steps):
        s.newton_step(case.cfg.cfl)
    return time.perf_counter() - t0
