"""The multicolour sweep the GPU runs (split at the diagonal, explicit
diagonal inverses, the colour-0 product fused into the last pass), restated
in numpy (oracle/colour_sgs.py) and checked on the CPU against the
reference build's sequential SGS and SpMV on colour-ordered matrices made
from the reference's own Jacobian.

Tolerance 1e-10: the explicit inverse of a diagonal block instead of its
pivoted LU changes the rounding by the block's condition number times the
FP64 unit roundoff."""
import numpy as np
import pytest

import colour_sgs as CS
from conftest import rel_err


def _ref_matrix(cb, refh, make, cfl=7.5):
    case = make(cb)
    case.cfg.jacobian = cb.JAC_REFERENCE
    mesh = cb.HostMesh(case.spec)
    ref = refh.RefSolver(mesh, case.cfg, case.bcs)
    ref.set_state(cb.cases.perturbed_state(case, mesh.n_cells))
    ref.stages()
    _, vals = ref.jacobian(cfl)
    off, nb = refh.connectivity(mesh, 1)
    n = mesh.n_cells
    row_ptr = np.zeros(n + 1, dtype=np.int32)
    cols = []
    for c in range(n):
        cols.extend(sorted([c] + list(nb[off[c]:off[c + 1]])))
        row_ptr[c + 1] = len(cols)
    return row_ptr, np.array(cols, dtype=np.int32), vals


@pytest.mark.parametrize("name,make", [
    ("ramp", lambda cb: cb.cases.ramp(scale=2)),
    ("bump_tets", lambda cb: cb.cases.bump(scale=16, mixed=False)),
])
def test_split_sweep_and_fused_product_match_the_reference(cb, refh, name, make):
    row_ptr, cols, vals = _ref_matrix(cb, refh, make)
    rp, cl, vb, off, _ = CS.colour_order(row_ptr, cols, vals, 5)
    n = len(rp) - 1
    assert off[-1] == n and len(off) - 1 >= 2
    if name == "bump_tets":
        assert len(off) - 1 > 2  # tets need more than two colours
    r = np.random.default_rng(5).standard_normal(n * 5)
    z, az = CS.split_sweep_with_product(rp, cl, vb, 5, off, r)
    assert rel_err(z, refh.sgs_apply(rp, cl, vb, 5, r)) < 1e-10
    assert rel_err(az, refh.bsr_spmv(rp, cl, vb, 5, z)) < 1e-12


def test_recolouring_a_colour_ordered_matrix_keeps_the_colours(cb, refh):
    """The solver colours the matrix, stores it colour by colour and colours
    it again for the sweep: the greedy colouring of the permuted matrix must
    give the same contiguous, ascending colour ranges (the premise of the
    split sweep and the fused product)."""
    row_ptr, cols, vals = _ref_matrix(cb, refh, lambda cb: cb.cases.bump(scale=16, mixed=False))
    rp, cl, _, off, _ = CS.colour_order(row_ptr, cols, vals, 5)
    again = CS.greedy_colours(rp, cl)
    expect = np.repeat(np.arange(len(off) - 1), np.diff(off))
    assert np.array_equal(again, expect)
