"""Numpy restatement of the multicolour SGS apply that the GPU runs on a
colour-ordered matrix (test infrastructure only; the checker of the
algorithm in distributed-cfd-solver_b200/csrc/kernels_linalg.cu and
BsrSystem::sgs_apply_spmv in csrc/solver.cpp).

On a matrix whose rows are ordered colour by colour (a greedy colouring in
row order, colours ascending), the sweep is:
  forward, colours ascending:  y_i = D_i^-1 (r_i - sum_{j<i} A_ij y_j)
  backward, colours descending (the last colour already final):
      t_i = sum_{j>i} A_ij z_j,  z_i = y_i - D_i^-1 t_i
with D_i^-1 the explicit inverse of the diagonal block, and for colour 0
(swept last) the product (A z)_i = t_i + A_ii z_i formed in the same pass.
The reference's sequential SGS (bsr_sgs_sweep, natural row order, one
symmetric sweep from z = 0) is the same preconditioner on such a matrix:
rows of one colour do not couple.
"""
from __future__ import annotations

import numpy as np


def greedy_colours(row_ptr, cols):
    """Smallest colour not used by an already coloured neighbour, rows in
    order (BsrSystem::build_ordering, colour branch)."""
    n = len(row_ptr) - 1
    colour = np.full(n, -1, dtype=np.int64)
    for i in range(n):
        used = {int(colour[j]) for j in cols[row_ptr[i]:row_ptr[i + 1]] if j != i and colour[j] >= 0}
        c = 0
        while c in used:
            c += 1
        colour[i] = c
    return colour


def colour_order(row_ptr, cols, vals, bs):
    """The matrix with rows and columns permuted colour by colour (stable
    within a colour), columns sorted per row; returns (row_ptr, cols, vals,
    colour offsets, permutation new -> old)."""
    n = len(row_ptr) - 1
    colour = greedy_colours(row_ptr, cols)
    order = np.argsort(colour, kind="stable")
    new_of = np.empty(n, dtype=np.int64)
    new_of[order] = np.arange(n)
    blocks = np.asarray(vals).reshape(-1, bs, bs)
    rp = np.zeros(n + 1, dtype=np.int32)
    cl, vb = [], []
    for r, i in enumerate(order):
        ks = np.arange(row_ptr[i], row_ptr[i + 1])
        cn = new_of[cols[ks]]
        srt = np.argsort(cn)
        cl.extend(cn[srt])
        vb.append(blocks[ks[srt]])
        rp[r + 1] = len(cl)
    ncol = int(colour.max()) + 1
    off = np.zeros(ncol + 1, dtype=np.int64)
    for c in range(ncol):
        off[c + 1] = off[c] + int((colour == c).sum())
    return rp, np.asarray(cl, dtype=np.int32), np.concatenate(vb).ravel(), off, order


def split_sweep_with_product(row_ptr, cols, vals, bs, off, r):
    """z = M^-1 r by the split first sweep with explicit diagonal inverses,
    and A z with the colour-0 rows' product taken from the backward pass."""
    n = len(row_ptr) - 1
    A = np.asarray(vals, dtype=np.float64).reshape(-1, bs, bs)
    rr = np.asarray(r, dtype=np.float64).reshape(n, bs)
    diag = np.array([row_ptr[i] + int(np.searchsorted(cols[row_ptr[i]:row_ptr[i + 1]], i)) for i in range(n)])
    dinv = np.linalg.inv(A[diag])
    z = np.zeros((n, bs))
    ncol = len(off) - 1
    for c in range(ncol):                       # forward: lower blocks only
        for i in range(off[c], off[c + 1]):
            s = rr[i].copy()
            for k in range(row_ptr[i], diag[i]):
                s -= A[k] @ z[cols[k]]
            z[i] = dinv[i] @ s
    t = np.zeros((n, bs))
    for c in range(ncol - 2, -1, -1):           # backward: upper blocks only
        for i in range(off[c], off[c + 1]):
            for k in range(diag[i] + 1, row_ptr[i + 1]):
                t[i] += A[k] @ z[cols[k]]
            z[i] = z[i] - dinv[i] @ t[i]
    az = np.zeros((n, bs))
    for i in range(n):
        if i < off[1]:                          # colour 0: every off-diagonal block is in t
            az[i] = t[i] + A[diag[i]] @ z[i]
        else:
            for k in range(row_ptr[i], row_ptr[i + 1]):
                az[i] += A[k] @ z[cols[k]]
    return z.ravel(), az.ravel()
