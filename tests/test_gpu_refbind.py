"""The GPU adapters behind the reference's own interfaces
(distributed-cfd-solver_b200/refbind/cfdg_reference_adapters.hpp), driven by
the reference's own code: its BiCGSTAB with GpuSgs / GpuBsrOperator, the
GpuBiCGSTAB solver, GpuGradient through GradientOperator::apply_set, and
the reference Solver<...>::run loop with the GpuBackwardEuler time policy,
each against the same reference call with its CPU classes.  Tolerances as
the stage tests: SGS (level order) and operator paths 1e-10 on the Krylov
solution of a tightly solved system, gradients 1e-11, Newton iterates 1e-8."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refbind():
    import refbind as rb
    if not rb.available():
        pytest.skip("oracle/_ref/librefbind.so not built")
    return rb


@pytest.fixture(scope="module")
def ramp_system(cb, refh):
    case = cb.cases.ramp()
    case.cfg.jacobian = cb.JAC_REFERENCE
    mesh = cb.HostMesh(case.spec)
    ref = refh.RefSolver(mesh, case.cfg, case.bcs)
    ref.set_state(cb.cases.perturbed_state(case, mesh.n_cells))
    st = ref.stages()
    _, vals = ref.jacobian(5.0)
    off, val = refh.connectivity(mesh, 1)
    n = mesh.n_cells
    row_ptr = [0]
    cols = []
    for i in range(n):
        row = sorted([i] + list(val[off[i]:off[i + 1]]))
        cols += row
        row_ptr.append(len(cols))
    b = -np.ascontiguousarray(st["res"].reshape(5, n).T).ravel()
    return np.array(row_ptr), np.array(cols), vals, b


@pytest.mark.parametrize("mode", [1, 2, 3], ids=["ref_bicgstab+gpu_sgs", "ref_bicgstab+gpu_operator", "gpu_bicgstab"])
def test_reference_krylov_with_gpu_adapters(refbind, ramp_system, mode):
    row_ptr, cols, vals, b = ramp_system
    x_ref, r_ref = refbind.bicgstab(row_ptr, cols, vals, 5, b, 0, rel_tol=1e-10, max_it=200)
    x, r = refbind.bicgstab(row_ptr, cols, vals, 5, b, mode, rel_tol=1e-10, max_it=200)
    assert r_ref["status"] == 0 and r["status"] == 0
    assert abs(r["iterations"] - r_ref["iterations"]) <= 1
    assert rel_err(x, x_ref) < 1e-8


def test_gpu_gmres_behind_the_iterative_solver_interface(refbind, ramp_system):
    """GpuGmres through linalg::IterativeSolver (GpuBsrOperator, GpuSgs):
    the reference BiCGSTAB's solution of the same tightly solved system."""
    row_ptr, cols, vals, b = ramp_system
    x_ref, r_ref = refbind.bicgstab(row_ptr, cols, vals, 5, b, 0, rel_tol=1e-10, max_it=200)
    x, r = refbind.bicgstab(row_ptr, cols, vals, 5, b, 4, rel_tol=1e-10, max_it=400)
    assert r_ref["status"] == 0 and r["status"] == 0
    assert rel_err(x, x_ref) < 1e-8


@pytest.mark.parametrize("stencil", [2, 3], ids=["face", "node"])
def test_gpu_gradient_operator(cb, refbind, stencil):
    case = cb.cases.plate(scale=8)
    mesh = cb.HostMesh(case.spec)
    rng = np.random.default_rng(3)
    q = rng.standard_normal((7, mesh.n_cells))
    g_ref = refbind.gradient(mesh, stencil, q, gpu=False)
    g = refbind.gradient(mesh, stencil, q, gpu=True)
    for v in range(7):
        assert rel_err(g[v], g_ref[v]) < 1e-11


@pytest.mark.parametrize("name", ["ramp", "plate"])
def test_reference_solver_loop_with_gpu_time_policy(cb, refbind, name):
    case = cb.cases.ramp() if name == "ramp" else cb.cases.plate(scale=8)
    case.cfg.jacobian = cb.JAC_REFERENCE
    case.cfg.sgs_ordering = cb.SGS_LEVEL
    case.cfg.cfl = 5.0
    case.cfg.max_iterations = 4
    mesh = cb.HostMesh(case.spec)
    U_cpu = refbind.run(mesh, case.cfg, case.bcs, gpu=False)
    U_gpu = refbind.run(mesh, case.cfg, case.bcs, gpu=True)
    assert np.all(np.isfinite(U_gpu))
    assert rel_err(U_gpu, U_cpu, mesh.n_cells) < 1e-8
