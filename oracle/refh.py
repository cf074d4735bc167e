"""ctypes binding of oracle/_ref/libcfdref.so (the reference solver built from
its own sources with the single-rank MPI shim, see ref_harness.cpp).

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg use it, as the checker.  It takes the same cfdg_mesh_host /
cfdg_config / cfdg_bc_desc structures as the product library.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libcfdref.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_L = None


def available() -> bool:
    return REF_LIB.exists()


def _lib():
    global _L
    if _L is None:
        if not REF_LIB.exists():
            raise RuntimeError(f"{REF_LIB} missing: run make -C {HERE} ref")
        L = C.CDLL(str(REF_LIB))
        L.refh_compute_geometry.argtypes = [C.c_void_p, _dp, _dp]
        L.refh_validate.argtypes = [C.c_void_p]
        L.refh_connectivity.argtypes = [C.c_void_p, C.c_int, _ip, _ip, C.c_int64]
        L.refh_connectivity.restype = C.c_int64
        L.refh_wall_distance.argtypes = [C.c_void_p, C.POINTER(C.c_uint8), C.c_int, C.c_int, C.c_double, _dp]
        L.refh_create.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]
        L.refh_destroy.argtypes = [C.c_void_p]
        L.refh_nnzb.argtypes = [C.c_void_p]
        L.refh_nnzb.restype = C.c_int64
        L.refh_set_state.argtypes = [C.c_void_p, _dp, C.c_int64]
        L.refh_get_state.argtypes = [C.c_void_p, _dp, C.c_int64]
        L.refh_stages.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.refh_jacobian.argtypes = [C.c_void_p, C.c_double, _dp, _dp]
        L.refh_newton_step.argtypes = [C.c_void_p, C.c_double, _dp]
        L.refh_freeze_limiter.argtypes = [C.c_void_p, C.c_int]
        L.refh_mesh_generate.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        L.refh_mesh_view.argtypes = [C.c_void_p, C.c_void_p]
        L.refh_mesh_free.argtypes = [C.c_void_p]
        L.refh_run_unsteady.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, _dp]
        L.refh_write_vtu.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p]
        L.refh_bsr_spmv.argtypes = [C.c_int, C.c_int, _ip, _ip, _dp, _dp, _dp, C.c_double, C.c_double]
        L.refh_sgs_apply.argtypes = [C.c_int, C.c_int, _ip, _ip, _dp, _dp, _dp, C.c_int]
        L.refh_bicgstab.argtypes = [C.c_int, C.c_int, _ip, _ip, _dp, C.c_int, C.c_double, C.c_double, C.c_int, _dp,
                                    _dp, C.POINTER(C.c_int), C.POINTER(C.c_int), _dp, _dp]
        _L = L
    return _L


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def compute_geometry(mesh):
    """Reference compute_mesh_geometry on the topology of `mesh` (a HostMesh)."""
    n, nf = mesh.n_cells, mesh.n_faces
    cell = np.zeros(4 * n)
    face = np.zeros(7 * nf)
    _lib().refh_compute_geometry(C.byref(mesh.view), _d(cell), _d(face))
    return cell.reshape(4, n), face.reshape(7, nf)


def validate(mesh) -> None:
    _lib().refh_validate(C.byref(mesh.view))


def connectivity(mesh, kind: int):
    n = mesh.n_cells
    off = np.zeros(n + 1, dtype=np.int32)
    cnt = _lib().refh_connectivity(C.byref(mesh.view), kind, _i(off), None, 0)
    val = np.zeros(max(cnt, 1), dtype=np.int32)
    _lib().refh_connectivity(C.byref(mesh.view), kind, _i(off), _i(val), cnt)
    return off, val[:cnt]


def wall_distance(mesh, wall_patches, max_sweeps=100000, rel_tol=0.0):
    """Reference graph wall distance (face-neighbour stencil) to the patches in
    `wall_patches`; the defaults relax to the exact fixed point."""
    npatch = int(mesh.view.n_patches)
    mask = np.zeros(max(npatch, 1), dtype=np.uint8)
    for p in wall_patches:
        mask[p] = 1
    out = np.zeros(mesh.n_cells)
    _lib().refh_wall_distance(C.byref(mesh.view), mask.ctypes.data_as(C.POINTER(C.c_uint8)), npatch, max_sweeps,
                              rel_tol, _d(out))
    return out


_up = C.POINTER(C.c_uint8)


class MeshHost(C.Structure):
    """cfdg_mesh_host of include/cfdg.h (the view RefMesh hands out)."""
    _fields_ = [("n_cells", C.c_int32), ("n_faces", C.c_int32), ("n_inner_faces", C.c_int32),
                ("n_nodes", C.c_int32), ("n_patches", C.c_int32),
                ("cell_type", _up), ("cell_nodes_offsets", _ip), ("cell_nodes", _ip),
                ("node_x", _dp), ("node_y", _dp), ("node_z", _dp),
                ("cell_centroid_x", _dp), ("cell_centroid_y", _dp), ("cell_centroid_z", _dp), ("cell_volume", _dp),
                ("face_owner", _ip), ("face_neigh", _ip), ("face_patch", _ip),
                ("face_nodes_offsets", _ip), ("face_nodes", _ip),
                ("face_centroid_x", _dp), ("face_centroid_y", _dp), ("face_centroid_z", _dp),
                ("face_normal_x", _dp), ("face_normal_y", _dp), ("face_normal_z", _dp), ("face_area", _dp)]


class RefMesh:
    """A benchmark mesh built by the reference's own preprocessing pipeline
    (build_faces -> migrate_local_mesh at one rank -> compute_mesh_geometry
    -> reorder_local_mesh(RCM) -> validate, as apps/mesh_partition.cpp runs
    it) from the seeded synthetic generator's cells, nodes and boundary
    patches.  Same interface as the product's HostMesh (`view`, `n_cells`,
    `n_faces`, `n_inner`), so RefSolver and the C restatement take it."""

    def __init__(self, spec):
        h = C.c_void_p()
        if _lib().refh_mesh_generate(C.byref(spec), C.byref(h)) != 0:
            raise ValueError("invalid mesh spec")
        self._h = h
        self.spec = spec
        self.view = MeshHost()
        _lib().refh_mesh_view(self._h, C.byref(self.view))

    def close(self):
        if getattr(self, "_h", None):
            _lib().refh_mesh_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_cells(self) -> int:
        return self.view.n_cells

    @property
    def n_faces(self) -> int:
        return self.view.n_faces

    @property
    def n_inner(self) -> int:
        return self.view.n_inner_faces


class RefSolver:
    """Reference solver over one mesh/config (5 mean-flow variables)."""

    def __init__(self, mesh, cfg, bcs):
        from ctypes import byref
        self.n = mesh.n_cells
        self.nt = mesh.n_cells + mesh.n_faces - mesh.n_inner
        arr = (type(bcs[0]) * len(bcs))(*bcs)
        h = C.c_void_p()
        _lib().refh_create(byref(mesh.view), byref(cfg), arr, len(bcs), byref(h))
        self._h = h
        self.nnzb = int(_lib().refh_nnzb(self._h))

    def close(self):
        if getattr(self, "_h", None):
            _lib().refh_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(5, -1)
        _lib().refh_set_state(self._h, _d(U), U.shape[1])

    def get_state(self):
        U = np.zeros((5, self.n))
        _lib().refh_get_state(self._h, _d(U), self.n)
        return U

    def stages(self):
        n, nt = self.n, self.nt
        q, grad, phi, res, lam = np.zeros(5 * nt), np.zeros(15 * nt), np.zeros(5 * n), np.zeros(5 * n), np.zeros(n)
        _lib().refh_stages(self._h, _d(q), _d(grad), _d(phi), _d(res), _d(lam))
        return {"q": q, "grad": grad, "phi": phi, "res": res, "lam": lam}

    def jacobian(self, cfl):
        alpha = np.zeros(self.n)
        vals = np.zeros(self.nnzb * 25)
        _lib().refh_jacobian(self._h, cfl, _d(alpha), _d(vals))
        return alpha, vals

    def write_vtu(self, outdir, stem):
        """The reference's write_solution_vtu of the Solver's current state."""
        _lib().refh_write_vtu(self._h, str(outdir).encode(), stem.encode())

    def freeze_limiter(self, frozen=True):
        """Keep the Solver's limiter values of the last evaluation (the
        library's limiter freeze, applied through the reconstruction policy)."""
        _lib().refh_freeze_limiter(self._h, 1 if frozen else 0)

    def newton_step(self, cfl):
        l2 = np.zeros(5)
        _lib().refh_newton_step(self._h, cfl, _d(l2))
        return l2


def run_unsteady(mesh, cfg, bcs):
    """The reference Solver with BackwardEuler and UnsteadyMode<cfg.bdf_order>
    run from init_fields: cfg.max_time_steps physical steps of
    cfg.dt_physical, cfg.max_iterations sub-iterations each (fewer if the
    reference monitor drops below cfg.residual_tolerance).  Returns U (5 x n)."""
    U = np.zeros((5, mesh.n_cells))
    arr = (type(bcs[0]) * len(bcs))(*bcs)
    _lib().refh_run_unsteady(C.byref(mesh.view), C.byref(cfg), arr, len(bcs), _d(U))
    return U


def bsr_spmv(row_ptr, cols, vals, bs, x, y=None, alpha=1.0, beta=0.0):
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros_like(x) if y is None else np.array(y, dtype=np.float64, copy=True)
    _lib().refh_bsr_spmv(len(row_ptr) - 1, bs, _i(row_ptr), _i(cols), _d(vals), _d(x), _d(y), alpha, beta)
    return y


def sgs_apply(row_ptr, cols, vals, bs, r, sweeps=1):
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    r = np.ascontiguousarray(r, dtype=np.float64)
    z = np.zeros_like(r)
    _lib().refh_sgs_apply(len(row_ptr) - 1, bs, _i(row_ptr), _i(cols), _d(vals), _d(r), _d(z), sweeps)
    return z


def bicgstab(row_ptr, cols, vals, bs, b, x0=None, precond=1, rel_tol=1e-8, abs_tol=1e-30, max_it=500):
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
    it, st = C.c_int(), C.c_int()
    r0, rf = np.zeros(1), np.zeros(1)
    _lib().refh_bicgstab(len(row_ptr) - 1, bs, _i(row_ptr), _i(cols), _d(vals), precond, rel_tol, abs_tol, max_it,
                         _d(x), _d(b), C.byref(it), C.byref(st), _d(r0), _d(rf))
    return x, {"iterations": it.value, "status": st.value, "initial": float(r0[0]), "final": float(rf[0])}
