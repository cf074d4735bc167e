"""The nu_tilde row of the 6x6 Picard Jacobian (entries [5][5]: upwind
convection, compact diffusion, the boundary ghosts' dependence on the owner,
the destruction derivative) against central finite differences of the
oracle's own nu_tilde residual in rho*nu_tilde, mean flow frozen.

The Picard row drops the diffusion coefficient's derivative, the averaged
cell gradients in the face gradient, the production derivative and f_w's
dependence on nu_tilde.  In a uniform free stream with uniform nu_tilde on
the plate's box cells (face-to-cell vectors along the face normals) every
dropped term vanishes: the face gradient is (nu_R - nu_L)/|d|, the strain is
zero (production at its floor, r clipped so f_w is constant) and the cb2 and
coefficient terms are second order in the perturbation.  The Picard row is
then the exact derivative, and the finite differences must reproduce every
entry: wall, inflow, outflow and symmetry faces included.  (The benchmark
plate's jittered grid lines tilt the faces slightly; there the dropped
averaged-gradient terms show up at 1e-6 of the row scale.)"""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def port():
    import port as p
    if not p.available():
        pytest.skip("oracle/_ref/liboracle.so not built")
    return p


def test_nu_tilde_jacobian_row_is_the_derivative_of_the_residual(cb, port):
    case = cb.cases.sa_plate(scale=16, mixed=False)
    case.spec.jitter = 0.0  # box cells: every face-to-cell vector along the face normal
    mesh = cb.HostMesh(case.spec)
    n = mesh.n_cells
    s = port.PortSolver(mesh, case.cfg, case.bcs)
    U0 = cb.cases.freestream_state(case, n)
    s.set_state(U0)
    s.stages()
    alpha, vals = s.jacobian(5.0)
    rp, cols = s.structure()
    vals = vals.reshape(-1, 6, 6)
    rng = np.random.default_rng(4)
    # every boundary-adjacent cell kind plus a random interior sample
    a = mesh.arrays()
    nb_owner = a["face_owner"][mesh.n_inner:]
    picks = np.unique(np.concatenate([nb_owner[:: max(1, len(nb_owner) // 40)], rng.choice(n, 40, replace=False)]))
    worst = 0.0
    for j in picks:
        h = 1e-6 * U0[5, j]
        col = []
        for sgn in (1.0, -1.0):
            U = U0.copy()
            U[5, j] += sgn * h
            s.set_state(U)
            col.append(s.stages()["res"].reshape(6, n)[5])
        fd = (col[0] - col[1]) / (2 * h)
        # rows i whose block column j is stored: the [5][5] entry
        expect = np.zeros(n)
        for i in range(n):
            for k in range(rp[i], rp[i + 1]):
                if cols[k] == j:
                    expect[i] = vals[k, 5, 5] - (alpha[i] if i == j else 0.0)
        scale = np.abs(expect).max()
        err = np.abs(fd - expect).max() / scale
        worst = max(worst, err)
        # nothing outside the stored stencil
        assert np.all(fd[expect == 0.0] == 0.0) or np.abs(fd[expect == 0.0]).max() < 1e-8 * scale
    assert worst < 1e-6, worst
