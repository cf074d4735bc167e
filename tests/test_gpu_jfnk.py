"""Jacobian-free Newton-Krylov operator (CFDG_NEWTON_JACOBIAN_FREE) on the
GPU, checked through the library's own residual.

1. A Jacobian-free linear solve solves the Jacobian-free system.  For its
   update du, r = alpha du + (R(U + h du) - R(U)) / h + R(U), with R
   evaluated by the library at U and at U + h du (h by the product's own
   rule: no variable moves by more than 1e-7 of its RMS), is below the
   solve's tolerance plus the finite-difference error, relative to
   ||R(U)||.  The Picard update of the same state leaves a much larger r:
   its first-order matrix omits the reconstruction's dependence on the
   neighbours' neighbours.
2. The product is the FP64 residual whatever the matrix precision: with the
   FP32 matrix (mixed precision) only the preconditioner changes and the
   same bound holds.
3. The compression ramp (4,096 cells) run to a 1e-8 drop with the
   Jacobian-free operator after the limiter freeze lands on the reference
   build's converged field of the same frozen problem (FP64 level-sweep
   iterates before the freeze) to 1e-6 relative L2 on rho, u, v, p, in fewer
   Newton iterations than the Picard run.
4. Switched evolution relaxation raises the CFL past cfl_max and lands on
   the same converged field.
5. Out-of-range Jacobian-free options are refused at solver creation.
"""
import numpy as np
import pytest

from converged import converge_host, field_errors

pytestmark = pytest.mark.gpu


def _jf_system_residual(cb, precision, newton_operator):
    case = cb.cases.ramp()
    case.cfg.newton_operator = newton_operator
    case.cfg.jf_rel_tol = 1e-8
    case.cfg.jf_max_iterations = 300
    case.cfg.lin_rel_tol = 1e-8
    case.cfg.lin_max_iterations = 300
    case.cfg.precision = precision
    case.cfg.pre_freeze = cb.PREFREEZE_CONFIGURED
    mesh = cb.HostMesh(case.spec)
    n = mesh.n_cells
    U0 = np.asarray(cb.cases.perturbed_state(case, n)).reshape(5, n).copy()
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        s.set_state(U0)
        s.evaluate_residual()       # limiter values of U0 ...
        s.freeze_limiter(True)      # ... frozen: R is differentiable
        s.evaluate_residual()
        s.compute_dt(20.0)
        s.assemble_jacobian()
        kr = s.linear_solve()
        du = s.get(cb.FIELD_DU).reshape(n, 5).T.copy()
        R0 = s.get(cb.FIELD_RES).reshape(5, n).copy()
        alpha = s.get(cb.FIELD_ALPHA).copy()
        su = np.sqrt((U0 ** 2).mean(axis=1))
        h = 1e-7 / (np.abs(du).max(axis=1) / su).max()
        s.set_state(U0 + h * du)
        s.evaluate_residual()
        R1 = s.get(cb.FIELD_RES).reshape(5, n).copy()
    r = alpha * du + (R1 - R0) / h + R0
    return float(np.linalg.norm(r) / np.linalg.norm(R0)), kr


def test_jacobian_free_solve_solves_the_jacobian_free_system(cb):
    rel_jf, kr = _jf_system_residual(cb, 0, cb.NEWTON_JACOBIAN_FREE)
    rel_picard, _ = _jf_system_residual(cb, 0, cb.NEWTON_PICARD)
    assert kr.status == cb.KRYLOV_CONVERGED, kr.status
    assert rel_jf < 1e-5, rel_jf
    assert rel_picard > 100 * rel_jf, (rel_picard, rel_jf)


def test_jacobian_free_product_is_fp64_with_the_fp32_matrix(cb):
    rel_jf, kr = _jf_system_residual(cb, 1, cb.NEWTON_JACOBIAN_FREE)
    assert kr.status == cb.KRYLOV_CONVERGED, kr.status
    assert rel_jf < 1e-5, rel_jf


@pytest.fixture(scope="module")
def ramp_reference(cb, refh):
    case = cb.cases.ramp(iterations=2000)
    mesh = cb.HostMesh(case.spec)
    U0 = cb.cases.freestream_state(case, mesh.n_cells)
    U_ref, it = converge_host(cb, refh.RefSolver(mesh, case.cfg, case.bcs), case, U0)
    return mesh, U_ref, it


def _run(cb, mesh, newton_operator, precision=0):
    case = cb.cases.ramp(iterations=2000)
    case.cfg.sgs_ordering = cb.SGS_LEVEL
    case.cfg.newton_operator = newton_operator
    case.cfg.precision = precision
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        s.init_fields()
        r = s.run_steady()
        U = s.get(cb.FIELD_U).reshape(5, -1)
    assert r.converged and not r.blowup, (r.iterations, r.rel)
    return U, r


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_ramp_jacobian_free_converges_to_the_reference_field(cb, ramp_reference, precision):
    mesh, U_ref, it_ref = ramp_reference
    U, r = _run(cb, mesh, cb.NEWTON_JACOBIAN_FREE, precision)
    _, rp = _run(cb, mesh, cb.NEWTON_PICARD, precision)
    err = field_errors(U, U_ref)
    assert max(err.values()) < 1e-6, (err, r.iterations, it_ref)
    assert r.jacobian_free_steps > 0
    assert r.iterations < rp.iterations, (r.iterations, rp.iterations, r.picard_fallbacks)


def test_ser_raises_the_cfl_and_keeps_the_converged_field(cb, ramp_reference):
    """Switched evolution relaxation changes only the pseudo-time path: the
    CFL climbs above cfl_max after the ramp and the run lands on the
    reference's converged field of the same frozen problem."""
    mesh, U_ref, _ = ramp_reference
    case = cb.cases.ramp(iterations=2000)
    case.cfg.sgs_ordering = cb.SGS_LEVEL
    case.cfg.cfl_ser_max = 1000.0
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        s.init_fields()
        r = s.run_steady()
        U = s.get(cb.FIELD_U).reshape(5, -1)
    assert r.converged and not r.blowup
    assert r.cfl_last > case.cfg.cfl_max
    err = field_errors(U, U_ref)
    assert max(err.values()) < 1e-6, err


@pytest.mark.parametrize("field,value", [("newton_operator", 7), ("jf_accept", 0.0), ("jf_restart", 0),
                                         ("jf_krylov", 5), ("jf_eps", 0.0)])
def test_jacobian_free_options_are_checked(cb, field, value):
    case = cb.cases.ramp()
    case.cfg.newton_operator = cb.NEWTON_JACOBIAN_FREE
    setattr(case.cfg, field, value)
    mesh = cb.HostMesh(case.spec)
    with pytest.raises(cb.CfdgError):
        cb.Solver(mesh, case.cfg, case.bcs)
