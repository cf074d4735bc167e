"""Failure detection through status codes, injected on the host (no GPU
fault): non-finite state, singular diagonal block, broken mesh, Krylov
breakdown and iteration limits.  Every failing call returns a status and
leaves the context usable for the next call."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _eye_bsr(cb, n=12, bs=5, scale=1.0):
    rp = np.arange(n + 1, dtype=np.int32)
    cols = np.arange(n, dtype=np.int32)
    A = cb.Bsr(rp, cols, bs)
    A.set_values(np.tile(scale * np.eye(bs).ravel(), n))
    return A


def test_identity_breakdown_matches_reference_semantics(cb):
    # s = 0 after the first half-step -> t.t == 0 -> Diverged, x untouched
    # (bicgstab.cpp:138-141), exactly as the reference and the oracle do.
    A = _eye_bsr(cb)
    b = np.arange(1.0, 61.0)
    x, info = A.bicgstab(b, precond=cb.PC_NONE, rel_tol=1e-12)
    assert info.status == cb.KRYLOV_DIVERGED and info.iterations == 1
    assert np.all(x == 0.0)


def test_zero_rhs_and_max_iterations(cb):
    A = _eye_bsr(cb, scale=2.0)
    x, info = A.bicgstab(np.zeros(60), precond=cb.PC_NONE)
    assert info.status == cb.KRYLOV_CONVERGED and info.iterations == 0
    x, info = A.bicgstab(np.ones(60), precond=cb.PC_NONE, max_it=0)
    assert info.status == cb.KRYLOV_MAX_ITERATIONS and info.iterations == 0


def test_gmres_edge_cases(cb):
    # identity: one iteration, exact; zero right-hand side: no iteration;
    # max_it = 0: no iteration, max-iterations status
    A = _eye_bsr(cb, scale=2.0)
    b = np.arange(1.0, 61.0)
    x, info = A.gmres(b, precond=cb.PC_NONE, rel_tol=1e-12)
    assert info.status == cb.KRYLOV_CONVERGED and info.iterations == 1
    assert np.allclose(x, b / 2.0, rtol=1e-14, atol=0.0)
    x, info = A.gmres(np.zeros(60), precond=cb.PC_NONE)
    assert info.status == cb.KRYLOV_CONVERGED and info.iterations == 0
    x, info = A.gmres(np.ones(60), precond=cb.PC_NONE, max_it=0)
    assert info.status == cb.KRYLOV_MAX_ITERATIONS and info.iterations == 0
    with pytest.raises(cb.CfdgError):
        A.gmres(np.ones(60), precond=cb.PC_NONE, restart=0)


def test_singular_diagonal_block_reported(cb):
    n, bs = 8, 5
    rp = np.arange(n + 1, dtype=np.int32)
    A = cb.Bsr(rp, np.arange(n, dtype=np.int32), bs)
    vals = np.tile(np.eye(bs).ravel(), n)
    vals[3 * 25: 4 * 25] = 0.0  # block row 3 singular
    A.set_values(vals)
    with pytest.raises(cb.CfdgError) as e:
        A.sgs_setup(cb.SGS_COLOR, 1)
    assert e.value.status == cb.ERR_SINGULAR and "row 3" in str(e.value)
    vals[3 * 25: 4 * 25] = np.eye(bs).ravel()
    A.set_values(vals)
    A.sgs_setup(cb.SGS_COLOR, 1)  # the handle stays usable
    assert np.allclose(A.sgs_apply(np.ones(n * bs)), 1.0)


def test_nonfinite_state_detected_as_blowup(cb):
    case = cb.cases.ramp(scale=4, iterations=5)
    mesh = cb.HostMesh(case.spec)
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        U = cb.cases.freestream_state(case, mesh.n_cells)
        U[4, 7] = np.nan
        s.set_state(U)
        r = s.run_steady()
        assert r.blowup == 1 and r.iterations == 1
        # the solver recovers with a clean state
        s.init_fields()
        st = s.newton_step(1.0)
        assert np.all(np.isfinite(st.l2[:5]))


def test_invalid_inputs_rejected(cb):
    case = cb.cases.ramp(scale=4)
    mesh = cb.HostMesh(case.spec)
    with pytest.raises(cb.CfdgError) as e:
        cb.Solver(mesh, case.cfg, case.bcs[:-1])  # patch without a boundary condition
    assert e.value.status == cb.ERR_INVALID
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        with pytest.raises(cb.CfdgError):
            s.compute_dt(-1.0)
        with pytest.raises(cb.CfdgError):
            s.get(99)
    with pytest.raises(cb.CfdgError):
        cb.Bsr([0, 1, 2], [1, 0], 5)  # rows without a diagonal block
