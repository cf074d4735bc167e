"""ctypes binding of oracle/_ref/librefbind.so: the reference's own
BiCGSTAB, gradient operators and Solver<...> loop run with the CPU classes
or with the GPU adapters of distributed-cfd-solver_b200/refbind plugged into
the same seams (refbind_harness.cpp).  Test infrastructure."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_ref" / "librefbind.so"
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_L = None


def available() -> bool:
    return LIB.exists()


def _lib():
    global _L
    if _L is None:
        L = C.CDLL(str(LIB))
        L.rb_bicgstab.argtypes = [C.c_int, C.c_int, _ip, _ip, _dp, _dp, _dp, C.c_int, C.c_double, C.c_int,
                                  C.POINTER(C.c_int), C.POINTER(C.c_int), _dp]
        L.rb_gradient.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp, C.c_int]
        L.rb_run.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int, _dp]
        _L = L
    return _L


def _d(a):
    return a.ctypes.data_as(_dp)


def bicgstab(row_ptr, cols, vals, bs, b, mode, rel_tol=1e-8, max_it=500):
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    cols = np.ascontiguousarray(cols, dtype=np.int32)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    it, st, rf = C.c_int(), C.c_int(), np.zeros(1)
    _lib().rb_bicgstab(len(row_ptr) - 1, bs, row_ptr.ctypes.data_as(_ip), cols.ctypes.data_as(_ip), _d(vals),
                       _d(b), _d(x), mode, rel_tol, max_it, C.byref(it), C.byref(st), _d(rf))
    return x, {"iterations": it.value, "status": st.value, "final": float(rf[0])}


def gradient(mesh, stencil, q, gpu):
    q = np.ascontiguousarray(q, dtype=np.float64)
    nv, n = q.shape
    g = np.zeros((nv, 3, n))
    _lib().rb_gradient(C.byref(mesh.view), stencil, nv, _d(q), _d(g), 1 if gpu else 0)
    return g


def run(mesh, cfg, bcs, gpu):
    n = mesh.n_cells
    U = np.zeros((5, n))
    arr = (type(bcs[0]) * len(bcs))(*bcs)
    _lib().rb_run(C.byref(mesh.view), C.byref(cfg), arr, len(bcs), 1 if gpu else 0, _d(U))
    return U
