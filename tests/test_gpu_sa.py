"""GPU parity of the Spalart-Allmaras path (6 variables, 6x6 BSR) against
the oracle restatement (oracle/cfd_oracle.c, pinned by tests/test_sa_cpu.py),
through the C ABI.

Tolerances (FP64): primitives 1e-13; gradients, eddy viscosity, residual
1e-11 relative to the largest magnitude of each variable; wall distance
1e-15; Jacobian 1e-9 per 6x6 block (diagonal sums cancel); Newton iterates
1e-8 with the level-scheduled SGS (the oracle's sweep order).
"""
import numpy as np
import pytest

import sa_fields as F
from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def port():
    import port as p
    if not p.available():
        pytest.skip("oracle/_ref/liboracle.so not built")
    return p


def _setup(cb, port, scale=8, mixed=False):
    case = cb.cases.sa_plate(scale=scale, mixed=mixed)
    case.cfg.sgs_ordering = cb.SGS_LEVEL
    mesh = cb.HostMesh(case.spec)
    U0 = cb.cases.perturbed_state(case, mesh.n_cells)
    gpu = cb.Solver(mesh, case.cfg, case.bcs)
    ora = port.PortSolver(mesh, case.cfg, case.bcs)
    gpu.set_state(U0)
    ora.set_state(U0)
    return case, mesh, U0, gpu, ora


def test_sa_stages(cb, port):
    case, mesh, U0, gpu, ora = _setup(cb, port)
    assert gpu.nvars == 6 and gpu.bs == 6
    st = ora.stages()
    gpu.evaluate_residual()
    n, nt = gpu.n_cells, gpu.n_total
    assert rel_err(gpu.get(cb.FIELD_WALLDIST), st["wall_dist"]) < 1e-15
    assert rel_err(gpu.get(cb.FIELD_Q), st["q"], nt) < 1e-13
    g = gpu.get(cb.FIELD_GRAD)
    assert rel_err(g[: 15 * nt], st["grad"], nt) < 1e-11
    gn = gpu.get(cb.FIELD_NU_GRAD).reshape(3, nt)[:, :n]
    assert rel_err(gn, st["nu_grad"].reshape(3, nt)[:, :n], n) < 1e-11
    assert rel_err(gpu.get(cb.FIELD_NU), st["nu"]) < 1e-14
    assert rel_err(gpu.get(cb.FIELD_MUT)[:n], st["mut"][:n]) < 1e-13
    res = gpu.get(cb.FIELD_RES)
    assert rel_err(res, st["res"], n) < 1e-11
    assert rel_err(gpu.get(cb.FIELD_LAM), st["lam"]) < 1e-12


def test_sa_jacobian(cb, port):
    case, mesh, U0, gpu, ora = _setup(cb, port)
    ora.stages()
    alpha_ref, vals_ref = ora.jacobian(7.5)
    gpu.evaluate_residual()
    gpu.compute_dt(7.5)
    gpu.assemble_jacobian()
    assert rel_err(gpu.get(cb.FIELD_ALPHA), alpha_ref) < 1e-13
    vals = gpu.get(cb.FIELD_JAC)
    assert vals.shape == vals_ref.shape
    assert rel_err(vals, vals_ref, 36) < 1e-9
    blk = vals.reshape(-1, 6, 6)
    # Picard: no coupling between the mean flow and nu_tilde
    assert np.all(blk[:, 5, :5] == 0.0) and np.all(blk[:, :5, 5] == 0.0)


def test_sa_newton_steps(cb, port):
    case, mesh, U0, gpu, ora = _setup(cb, port)
    for k, cfl in enumerate([1.0, 3.0, 10.0]):
        st = gpu.newton_step(cfl)
        l2_ref = ora.newton_step(cfl)
        assert rel_err(np.array(st.l2[:6]), l2_ref) < 1e-9, k
        U = gpu.get(cb.FIELD_U)
        assert rel_err(U, ora.get_state().ravel(), mesh.n_cells) < 1e-8, k
        assert U.reshape(6, -1)[5].min() >= 0.0


def test_sa_analytic_fields(cb, port):
    """The device residual reproduces the closed-form SA-1994 sources on the
    shear field (strain with full weight, f_w with cw3^6 in the denominator)."""
    case, h = F.uniform_case(cb, wall=True)
    mesh = cb.HostMesh(case.spec)
    a = mesh.arrays()
    xc, yc, V = a["cell_centroid_x"], a["cell_centroid_y"], a["cell_volume"]
    T, rho, gamma, nu0 = 288.15, 1.2, 1.0, 3.0e-3
    U, _ = F.state(case, mesh.n_cells, rho, T, lambda y: gamma * y, lambda x, y: nu0 + 0.0 * x, xc, yc)
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        s.set_state(U)
        s.evaluate_residual()
        r5 = s.get(cb.FIELD_RES).reshape(6, -1)[5] / V
        d = s.get(cb.FIELD_WALLDIST)
    exp = F.shear_sources_expected(rho, F.sutherland(T), nu0, gamma, d)
    m = F.interior(xc, yc, h, case.spec.lx, case.spec.ny * h)
    assert np.abs(r5[m] - exp[m]).max() / np.abs(exp[m]).max() < 1e-9


def test_sa_mixed_precision_tracks_fp64(cb):
    """FP32 Jacobian/SGS with FP64 residual and update: after the same
    Newton steps the state stays close to the all-FP64 path (the outer FP64
    residual acts as iterative refinement)."""
    outs = []
    for mixed in (False, True):
        case = cb.cases.sa_plate(scale=8, mixed=mixed)
        mesh = cb.HostMesh(case.spec)
        with cb.Solver(mesh, case.cfg, case.bcs) as s:
            s.init_fields()
            for k in range(12):
                st = s.newton_step(cb.cases.cfl_at(case.cfg, k + 1))
                assert np.all(np.isfinite(np.array(st.l2[:6])))
            outs.append(s.get(cb.FIELD_U))
    assert rel_err(outs[1], outs[0], outs[0].size // 6) < 1e-3


def test_sa_bitwise_determinism(cb):
    case = cb.cases.sa_plate(scale=8)
    mesh = cb.HostMesh(case.spec)
    U0 = cb.cases.perturbed_state(case, mesh.n_cells)
    outs = []
    for _ in range(2):
        with cb.Solver(mesh, case.cfg, case.bcs) as s:
            s.set_state(U0)
            for cfl in (1.0, 5.0):
                s.newton_step(cfl)
            outs.append(s.get(cb.FIELD_U))
    assert np.array_equal(outs[0], outs[1])
