"""Generates the golden fixtures of tests/golden/ from the reference solver
itself (oracle/_ref/libcfdref.so, built from the reference sources with the
single-rank MPI shim).  Run from the repository root:

    python tests/golden/make_golden.py

Each fixture holds, for one small seeded case: the perturbed input state,
the reference's stage outputs (primitives + BC ghosts, gradients + ghost
gradients, limiter, residual, spectral radius), the compute_dt alpha and
BSR Jacobian at CFL 7.5, and three reference Newton iterations (norms and
states) with the sequential SGS at CFL 1, 3, 10.
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import __graft_entry__ as ge  # noqa: E402
import refh  # noqa: E402

CASES = {
    "ramp": lambda cb: cb.cases.ramp(scale=4),
    "plate": lambda cb: cb.cases.plate(scale=16, jacobian=cb.JAC_REFERENCE),
    "bump": lambda cb: cb.cases.bump(scale=32, mixed=False),
}
CFLS = (1.0, 3.0, 10.0)


def main():
    cb = ge.load_package()
    out_dir = Path(__file__).resolve().parent
    for name, make in CASES.items():
        case = make(cb)
        case.cfg.sgs_ordering = cb.SGS_LEVEL
        mesh = cb.HostMesh(case.spec)
        U0 = cb.cases.perturbed_state(case, mesh.n_cells)
        ref = refh.RefSolver(mesh, case.cfg, case.bcs)
        ref.set_state(U0)
        st = ref.stages()
        alpha, jac = ref.jacobian(7.5)
        ref2 = refh.RefSolver(mesh, case.cfg, case.bcs)
        ref2.set_state(U0)
        l2s, Us = [], []
        for cfl in CFLS:
            l2s.append(ref2.newton_step(cfl))
            Us.append(ref2.get_state())
        np.savez_compressed(out_dir / f"{name}.npz", n_cells=mesh.n_cells, n_faces=mesh.n_faces,
                            n_inner=mesh.n_inner, U0=U0, q=st["q"], grad=st["grad"], phi=st["phi"], res=st["res"],
                            lam=st["lam"], alpha=alpha, jac=jac, cfls=np.array(CFLS), l2=np.array(l2s),
                            U=np.array(Us))
        print(name, mesh.n_cells, "cells")


if __name__ == "__main__":
    main()
