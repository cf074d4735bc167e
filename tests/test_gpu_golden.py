"""GPU path against the committed golden fixtures (made by the reference
solver, tests/golden/make_golden.py) through the C ABI; needs no reference
build on the GPU box."""
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_err

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = {
    "ramp": lambda cb: cb.cases.ramp(scale=4),
    "plate": lambda cb: cb.cases.plate(scale=16, jacobian=cb.JAC_REFERENCE),
    "bump": lambda cb: cb.cases.bump(scale=32, mixed=False),
}


@pytest.mark.parametrize("name", list(CASES))
def test_gpu_matches_golden(cb, name):
    g = np.load(GOLDEN / f"{name}.npz")
    case = CASES[name](cb)
    case.cfg.sgs_ordering = cb.SGS_LEVEL
    mesh = cb.HostMesh(case.spec)
    n = mesh.n_cells
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        nt = s.n_total
        s.set_state(g["U0"])
        s.evaluate_residual()
        assert rel_err(s.get(cb.FIELD_Q), g["q"], nt) < 1e-13
        assert rel_err(s.get(cb.FIELD_GRAD)[: 15 * nt], g["grad"], nt) < 1e-11
        assert rel_err(s.get(cb.FIELD_PHI), g["phi"]) < 1e-9
        assert rel_err(s.get(cb.FIELD_RES), g["res"], n) < 1e-11
        assert rel_err(s.get(cb.FIELD_LAM), g["lam"]) < 1e-12
        s.compute_dt(7.5)
        s.assemble_jacobian()
        assert rel_err(s.get(cb.FIELD_ALPHA), g["alpha"]) < 1e-13
        assert rel_err(s.get(cb.FIELD_JAC), g["jac"], 25) < 1e-9
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        s.set_state(g["U0"])
        for k, cfl in enumerate(g["cfls"]):
            st = s.newton_step(float(cfl))
            assert rel_err(np.array(st.l2[:5]), g["l2"][k]) < 1e-10
            assert rel_err(s.get(cb.FIELD_U), g["U"][k].ravel(), n) < 1e-10
