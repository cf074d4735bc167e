"""The oracle (plain-C restatement, oracle/cfd_oracle.c) pinned against the
golden fixtures made by the reference solver itself, and against the
reference build directly on larger cases.  CPU only."""
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_err

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = {
    "ramp": lambda cb: cb.cases.ramp(scale=4),
    "plate": lambda cb: cb.cases.plate(scale=16, jacobian=cb.JAC_REFERENCE),
    "bump": lambda cb: cb.cases.bump(scale=32, mixed=False),
}


@pytest.fixture(scope="module")
def port():
    import port as p
    if not p.available():
        pytest.skip("oracle/_ref/liboracle.so not built")
    return p


def _case(cb, name):
    case = CASES[name](cb)
    case.cfg.sgs_ordering = cb.SGS_LEVEL
    return case, cb.HostMesh(case.spec)


@pytest.mark.parametrize("name", list(CASES))
def test_golden_inputs_reproducible(cb, name):
    g = np.load(GOLDEN / f"{name}.npz")
    case, mesh = _case(cb, name)
    assert (mesh.n_cells, mesh.n_faces, mesh.n_inner) == (int(g["n_cells"]), int(g["n_faces"]), int(g["n_inner"]))
    assert np.array_equal(cb.cases.perturbed_state(case, mesh.n_cells), g["U0"])


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_matches_golden(cb, port, name):
    g = np.load(GOLDEN / f"{name}.npz")
    case, mesh = _case(cb, name)
    n, nt = mesh.n_cells, mesh.n_cells + mesh.n_faces - mesh.n_inner
    s = port.PortSolver(mesh, case.cfg, case.bcs)
    s.set_state(g["U0"])
    st = s.stages()
    assert rel_err(st["q"], g["q"], nt) < 1e-13
    assert rel_err(st["grad"], g["grad"], nt) < 1e-11
    assert rel_err(st["phi"], g["phi"]) < 1e-9
    assert rel_err(st["res"], g["res"], n) < 1e-11
    assert rel_err(st["lam"], g["lam"]) < 1e-12
    alpha, jac = s.jacobian(7.5)
    assert rel_err(alpha, g["alpha"]) < 1e-13
    assert rel_err(jac, g["jac"], 25) < 1e-9
    s2 = port.PortSolver(mesh, case.cfg, case.bcs)
    s2.set_state(g["U0"])
    for k, cfl in enumerate(g["cfls"]):
        l2 = s2.newton_step(float(cfl))
        assert rel_err(l2, g["l2"][k]) < 1e-10
        assert rel_err(s2.get_state().ravel(), g["U"][k].ravel(), n) < 1e-10


@pytest.mark.parametrize("name", ["ramp_full", "plate8"])
def test_oracle_matches_reference_build(cb, refh, port, name):
    case = cb.cases.ramp() if name == "ramp_full" else cb.cases.plate(scale=8, jacobian=cb.JAC_REFERENCE)
    case.cfg.sgs_ordering = cb.SGS_LEVEL
    mesh = cb.HostMesh(case.spec)
    U0 = cb.cases.perturbed_state(case, mesh.n_cells, seed=11)
    r, p = refh.RefSolver(mesh, case.cfg, case.bcs), port.PortSolver(mesh, case.cfg, case.bcs)
    r.set_state(U0)
    p.set_state(U0)
    for cfl in (2.0, 20.0):
        assert rel_err(p.newton_step(cfl), r.newton_step(cfl)) < 1e-10
        assert rel_err(p.get_state().ravel(), r.get_state().ravel(), mesh.n_cells) < 1e-10


def test_oracle_linalg_matches_reference_build(cb, refh, port):
    case = cb.cases.bump(scale=16, mixed=False)
    mesh = cb.HostMesh(case.spec)
    p = port.PortSolver(mesh, case.cfg, case.bcs)
    p.set_state(cb.cases.perturbed_state(case, mesh.n_cells))
    p.stages()
    _, vals = p.jacobian(4.0)
    rp, cols = p.structure()
    rng = np.random.default_rng(7)
    x = rng.standard_normal(mesh.n_cells * 5)
    y = rng.standard_normal(mesh.n_cells * 5)
    for a, b in [(1.0, 0.0), (-2.0, 0.5), (0.0, 2.0)]:
        assert rel_err(port.bsr_spmv(rp, cols, vals, 5, x, y, a, b), refh.bsr_spmv(rp, cols, vals, 5, x, y, a, b)) < 1e-14
    for sw in (1, 3):
        assert rel_err(port.sgs_apply(rp, cols, vals, 5, x, sw), refh.sgs_apply(rp, cols, vals, 5, x, sw)) < 1e-14
    for pc in (0, 1):
        sol, info = port.bicgstab(rp, cols, vals, 5, x, precond=pc, rel_tol=1e-9, max_it=300)
        sol_r, info_r = refh.bicgstab(rp, cols, vals, 5, x, precond=pc, rel_tol=1e-9, max_it=300)
        assert info["iterations"] == info_r["iterations"] and info["status"] == info_r["status"] == 0
        assert rel_err(sol, sol_r) < 1e-12


def test_oracle_krylov_edge_cases(port, refh):
    """Identity matrix (the A = I case of tests/linalg_test.cpp): in the
    reference the first iteration makes s = 0, so t.t == 0 trips the
    breakdown check (bicgstab.cpp:138-141) before x is updated: status
    Diverged after one iteration with x untouched.  The oracle reproduces
    that.  Zero right-hand side: converged with no iteration; max_it = 0:
    max-iterations status."""
    n, bs = 10, 3
    rp = np.arange(n + 1, dtype=np.int32)
    cols = np.arange(n, dtype=np.int32)
    vals = np.tile(np.eye(bs).ravel(), n)
    b = np.arange(1.0, n * bs + 1.0)
    x, info = port.bicgstab(rp, cols, vals, bs, b, precond=0, rel_tol=1e-12)
    x_r, info_r = refh.bicgstab(rp, cols, vals, bs, b, precond=0, rel_tol=1e-12)
    assert info == info_r
    assert info["iterations"] == 1 and info["status"] == 1 and np.array_equal(x, x_r)
    x, info = port.bicgstab(rp, cols, vals, bs, np.zeros(n * bs), precond=1)
    assert info["iterations"] == 0 and info["status"] == 0
    x, info = port.bicgstab(rp, cols, 2 * vals, bs, b, precond=0, max_it=0)
    assert info["status"] == 2


def test_oracle_frozen_limiter(cb, port):
    """The oracle's frozen limiter (the library's cfdg_solver_freeze_limiter):
    after freezing, a new state keeps the old limiter values; unfrozen, they
    are recomputed."""
    case, mesh = _case(cb, "ramp")
    s = port.PortSolver(mesh, case.cfg, case.bcs)
    U0 = cb.cases.perturbed_state(case, mesh.n_cells)
    s.set_state(U0)
    phi0 = s.stages()["phi"]
    assert phi0.min() < 1.0  # the perturbed ramp state is limited somewhere
    U1 = np.asarray(U0).reshape(5, -1) * (1.0 + 0.02 * np.sin(np.arange(mesh.n_cells)))
    s.freeze_limiter(True)
    s.set_state(U1)
    assert np.array_equal(s.stages()["phi"], phi0)
    s.freeze_limiter(False)
    assert not np.array_equal(s.stages()["phi"], phi0)


def _plate_bc_variant(cb, variant):
    """The 1/8 plate with one boundary condition swapped for a kind or mode
    the benchmark cases do not use."""
    case = cb.cases.plate(scale=8, jacobian=cb.JAC_REFERENCE)
    case.cfg.sgs_ordering = cb.SGS_LEVEL
    fs = case.extra
    if variant == "isothermal_wall":
        case.bcs[3] = cb.bc(3, cb.BC_NO_SLIP_WALL, t=310.0)
    elif variant == "heat_flux_wall":
        case.bcs[3] = cb.bc(3, cb.BC_NO_SLIP_WALL_HEAT_FLUX, tmp_grad=-40.0)
    elif variant == "inlet_mach_angles":
        case.bcs[0] = cb.bc(0, cb.BC_SUBSONIC_INLET, inflow_mode=cb.INFLOW_MACH_ANGLES, p=fs["p"], t=fs["T"],
                            mach=fs["mach"], alpha_deg=2.0, beta_deg=0.0)
    elif variant == "inlet_mach_direction":
        case.bcs[0] = cb.bc(0, cb.BC_SUBSONIC_INLET, inflow_mode=cb.INFLOW_MACH_DIRECTION, p=fs["p"], t=fs["T"],
                            mach=fs["mach"], direction=(0.99, 0.1, 0.0))
    elif variant == "farfield_top":
        case.bcs[2] = cb.bc(2, cb.BC_FARFIELD, p=fs["p"], t=fs["T"], velocity=(fs["u"], 0.0, 0.0))
    return case


@pytest.mark.parametrize("variant", ["isothermal_wall", "heat_flux_wall", "inlet_mach_angles",
                                     "inlet_mach_direction", "farfield_top"])
def test_oracle_boundary_variants_match_reference_build(cb, refh, port, variant):
    """Every boundary-condition kind and inflow mode the library accepts,
    beyond the benchmark cases' own: oracle stages and Newton iterates
    against the reference build."""
    case = _plate_bc_variant(cb, variant)
    mesh = cb.HostMesh(case.spec)
    U0 = cb.cases.perturbed_state(case, mesh.n_cells, seed=13)
    r, p = refh.RefSolver(mesh, case.cfg, case.bcs), port.PortSolver(mesh, case.cfg, case.bcs)
    r.set_state(U0)
    p.set_state(U0)
    sr, sp = r.stages(), p.stages()
    nt = mesh.n_cells + mesh.n_faces - mesh.n_inner
    assert rel_err(sp["q"], sr["q"], nt) < 1e-13
    assert rel_err(sp["res"], sr["res"], mesh.n_cells) < 1e-11
    for cfl in (2.0, 20.0):
        assert rel_err(p.newton_step(cfl), r.newton_step(cfl)) < 1e-10
        assert rel_err(p.get_state().ravel(), r.get_state().ravel(), mesh.n_cells) < 1e-10
