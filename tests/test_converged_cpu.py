"""The C restatement of the hot path against the reference build over a
whole convergence: the compression ramp (4,096 cells, FP64, the
reference's sequential SGS) run to a 1e-8 residual drop by both with the
CFL ramp and the limiter frozen at its end.  The two differ only in
rounding, and the switching limiter amplifies rounding until the freeze,
so the bar is on the converged fields (rho, u, v, p)."""
import numpy as np

from converged import converge_host, field_errors


def test_ramp_converged_restatement_equals_reference(cb, refh):
    import port
    case = cb.cases.ramp()
    mesh = cb.HostMesh(case.spec)
    U0 = cb.cases.freestream_state(case, mesh.n_cells)
    U_ref, it_ref = converge_host(cb, refh.RefSolver(mesh, case.cfg, case.bcs), case, U0)
    U_port, it_port = converge_host(cb, port.PortSolver(mesh, case.cfg, case.bcs), case, U0)
    assert abs(it_ref - it_port) <= 1
    err = field_errors(U_port, U_ref)
    assert max(err.values()) < 1e-9, err
