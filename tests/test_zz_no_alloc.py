"""cfdg_residual_norms_noalloc: the allocation-free residual norms for callers
that cannot allocate device memory (their pool owns the device budget, or
they run between solver kernels where cudaMalloc would synchronise).  Its
output must equal the solver's own cfdg_residual_norms, which uses library-
allocated scratch, on consecutive calls that share the static scratch.
Collected last so that a failure here leaves every other test already run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_norms_match_allocating_entry_point(cb):
    import torch

    L = cb.lib()
    case = cb.cases.plate(scale=8)
    mesh = cb.HostMesh(case.spec)
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        s.set_state(cb.cases.perturbed_state(case, mesh.n_cells))
        s.evaluate_residual()
        l2_ref = s.residual_norms()
        res = s.get(cb.FIELD_RES)
    n = mesh.n_cells
    dev = torch.from_numpy(res).to("cuda:0")
    dev2 = torch.from_numpy(3.0 * res[: 4 * n]).to("cuda:0")  # a second, different call
    torch.cuda.synchronize()
    out = np.zeros(6)
    rc = L.cfdg_residual_norms_noalloc(C.c_void_p(dev.data_ptr()), n, 5, None, out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == cb.OK, L.cfdg_last_error()
    assert np.allclose(out[:5], l2_ref, rtol=1e-12, atol=0.0)
    out2 = np.zeros(6)
    rc = L.cfdg_residual_norms_noalloc(C.c_void_p(dev2.data_ptr()), n, 4, None, out2.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == cb.OK, L.cfdg_last_error()
    assert np.allclose(out2[:4], 3.0 * l2_ref[:4], rtol=1e-12, atol=0.0)
    assert np.all(out2[4:] == 0.0)  # only nvars results are written
    # sizes beyond the static scratch are rejected before any GPU work
    rc = L.cfdg_residual_norms_noalloc(C.c_void_p(dev.data_ptr()), 4194305, 5, None, out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == cb.ERR_INVALID and b"4194304" in L.cfdg_last_error()
    rc = L.cfdg_residual_norms_noalloc(C.c_void_p(dev.data_ptr()), n, 7, None, out.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == cb.ERR_INVALID


def test_noalloc_norms_at_the_size_limit_on_a_side_stream(cb):
    # the largest accepted size (every one of the 16,384 x 6 partial slots in
    # use, next to the result slots) on a non-default stream, against numpy
    import torch

    L = cb.lib()
    n, nv = 4194304, 6
    rng = np.random.default_rng(11)
    res = rng.standard_normal((nv, n)) * np.array([1.0, 1e3, 1e-3, 5.0, 1e5, 1e-6])[:, None]
    expect = np.sqrt((res ** 2).sum(axis=1) / n)
    dev = torch.from_numpy(res.ravel()).to("cuda:0")
    side = torch.cuda.Stream(device="cuda:0")
    torch.cuda.synchronize()
    out = np.zeros(6)
    for _ in range(2):  # two calls in a row share the scratch
        rc = L.cfdg_residual_norms_noalloc(C.c_void_p(dev.data_ptr()), n, nv, C.c_void_p(side.cuda_stream),
                                           out.ctypes.data_as(C.POINTER(C.c_double)))
        assert rc == cb.OK, L.cfdg_last_error()
        assert np.allclose(out, expect, rtol=1e-12, atol=0.0)
