"""Solution output: the library's VTU files (fields formed on the GPU)
against the reference's io::vtk::write_solution_vtu of the same state on
the same mesh.  The geometry and topology sections must be identical text;
the CellData values (written with 11 significant digits) agree to 2e-10
relative, the last printed digit."""
import re

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sections(path):
    text = open(path).read()
    blocks = re.findall(r'<DataArray ([^>]*)>(.*?)</DataArray>', text, re.S)
    out = {}
    for head, body in blocks:
        name = re.search(r'Name="(\w+)"', head)
        out[name.group(1) if name else "points"] = body.split()
    return text, out


@pytest.mark.parametrize("name", ["ramp", "bump"])
def test_vtu_matches_reference_writer(cb, refh, tmp_path, name):
    case = cb.cases.ramp() if name == "ramp" else cb.cases.bump(scale=16, mixed=False)
    mesh = cb.HostMesh(case.spec)
    U = cb.cases.perturbed_state(case, mesh.n_cells)
    ref = refh.RefSolver(mesh, case.cfg, case.bcs)
    ref.set_state(U)
    ref.write_vtu(tmp_path / "ref", "state")
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        s.set_state(U)
        s.write_vtu(tmp_path / "gpu", "state")
    for suffix in (".pvtu",):
        assert (tmp_path / "gpu" / ("state" + suffix)).read_text() == (tmp_path / "ref" / ("state" + suffix)).read_text()
    _, g = _sections(tmp_path / "gpu" / "state_00000.vtu")
    _, r = _sections(tmp_path / "ref" / "state_00000.vtu")
    assert list(g) == list(r)
    for key in ("points", "connectivity", "offsets", "types", "rank"):
        assert g[key] == r[key], key
    for key in ("rho", "u", "v", "w", "pressure", "mach"):
        a, b = np.array(g[key], dtype=float), np.array(r[key], dtype=float)
        assert np.all(np.abs(a - b) <= 2e-10 * np.maximum(np.abs(b), 1e-300 + np.abs(b).max() * 1e-12)), key


def test_vtu_with_turbulence_fields(cb, tmp_path):
    case = cb.cases.sa_plate(scale=16, mixed=False)
    mesh = cb.HostMesh(case.spec)
    U = cb.cases.freestream_state(case, mesh.n_cells)
    with cb.Solver(mesh, case.cfg, case.bcs) as s:
        s.set_state(U)
        s.write_vtu(tmp_path, "sa")
    _, g = _sections(tmp_path / "sa_00000.vtu")
    assert "nu_tilde" in g and "mu_t" in g
    nu = np.array(g["nu_tilde"], dtype=float)
    assert np.allclose(nu, U[5] / U[0], rtol=1e-9)
    assert np.all(np.array(g["mu_t"], dtype=float) > 0)
