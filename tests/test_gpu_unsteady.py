"""Dual time stepping (BDF1 then BDF2, the reference's run_dual_time) on the
GPU against the reference Solver<..., BackwardEuler, UnsteadyMode<2>> from
the same initial state: the compression ramp and the 1/8 plate, three
physical steps of six sub-iterations each with the reference's sequential
SGS order.  Tolerance: the Newton iterates' 1e-8."""
import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu


def unsteady_case(cb, name, bdf):
    case = cb.cases.ramp() if name == "ramp" else cb.cases.plate(scale=8, jacobian=cb.JAC_REFERENCE)
    c = case.cfg
    c.time_mode = cb.TIME_UNSTEADY
    c.bdf_order = bdf
    c.dt_physical = 2.0e-5 if name == "ramp" else 1.0e-4
    c.max_time_steps = 3
    c.max_iterations = 6            # sub-iterations per physical step
    c.residual_tolerance = 1e-30    # run every sub-iteration
    c.cfl = c.cfl_max = 5.0
    c.cfl_ramp_iterations = 0
    c.convergence_monitor = 0       # the reference monitor
    c.limiter_freeze = 0
    c.sgs_ordering = cb.SGS_LEVEL
    c.jacobian = cb.JAC_REFERENCE
    return case


@pytest.mark.parametrize("name,bdf", [("ramp", 2), ("ramp", 1), ("plate", 2)])
def test_dual_time_matches_reference(cb, refh, name, bdf):
    case = unsteady_case(cb, name, bdf)
    mesh = cb.HostMesh(case.spec)
    U_ref = refh.run_unsteady(mesh, case.cfg, case.bcs)
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        s.init_fields()
        r = s.run_unsteady()
        U = s.get(cb.FIELD_U).reshape(5, -1)
    assert r.time_steps == 3 and r.subiterations_total == 18 and not r.blowup
    assert r.t_physical == pytest.approx(3 * case.cfg.dt_physical)
    U0 = cb.cases.freestream_state(case, mesh.n_cells)
    assert rel_err(U_ref, U0, mesh.n_cells) > 1e-6  # the flow moved
    assert rel_err(U, U_ref, mesh.n_cells) < 1e-8


def test_unsteady_mode_validation(cb):
    case = unsteady_case(cb, "ramp", 2)
    case.cfg.bdf_order = 3
    mesh = cb.HostMesh(case.spec)
    with pytest.raises(cb.CfdgError):
        cb.Solver(mesh, case.cfg, case.bcs)
    steady = cb.cases.ramp()
    with cb.Solver(mesh, steady.cfg, steady.bcs) as s:
        with pytest.raises(cb.CfdgError):
            s.run_unsteady()
