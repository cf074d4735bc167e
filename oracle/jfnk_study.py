"""CPU study on the oracle (test infrastructure, not part of the library):
the laminar plate's steady convergence with the Picard Jacobian (the
reference's backward-Euler Newton: the linear operator is the first-order
BSR matrix) against a Jacobian-free Newton-Krylov operator
v -> alpha v + (R(U + eps v) - R(U)) / eps on the full residual (eps: no
variable moves by more than 1e-7 of its RMS), both
right-preconditioned by SGS on the Picard matrix (oracle/cfd_oracle.c) and
solved by BiCGSTAB.  It measures what limits the plate's convergence; the
library itself has only the Picard path.

Usage (from the repository root):
  python oracle/jfnk_study.py --order second --method jfnk --iterations 600 \
      --cfl-max 1000 --scale 8 --freeze 150

--freeze k: freeze the MUSCL limiter at iteration k (the Jacobian-free
product needs a differentiable residual) and switch the JFNK operator on
from there; before it both methods are identical.  CFL: geometric ramp
1 -> 100 over 50 iterations, then switched evolution relaxation
CFL = 100 * (rel at the ramp's end / rel), capped at --cfl-max.
Prints one JSON line: every iterations/15 iterations the monitor
(max over mass, |momentum|, energy[, nu_tilde] of L2 / running maximum), the CFL, the
Krylov iterations since the last line and the last linear reduction.  A
Jacobian-free solve that does not reduce the linear residual is replaced by
the Picard step of the same iteration (counted in `picard_fallbacks`); a
Jacobian-free step is scaled so that density, energy and rho nu~ (against
its value plus 1e-3 of its RMS) change by at most 20% in any cell, and
rho nu~ is clipped at zero.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))


def bicgstab(op, prec, b, tol, maxit):
    """Right-preconditioned BiCGSTAB (the reference's algorithm, without the
    breakdown checks): returns (x, iterations, final |r| / |b|)."""
    x = np.zeros_like(b)
    r = b.copy()
    r0 = r.copy()
    p = r.copy()
    bn = np.linalg.norm(b)
    if bn == 0.0:
        return x, 0, 0.0
    rho = r0 @ r
    for k in range(1, maxit + 1):
        ph = prec(p)
        v = op(ph)
        alpha = rho / (r0 @ v)
        s = r - alpha * v
        sh = prec(s)
        t = op(sh)
        om = (t @ s) / (t @ t)
        x += alpha * ph + om * sh
        r = s - om * t
        if np.linalg.norm(r) <= tol * bn:
            return x, k, float(np.linalg.norm(r) / bn)
        rn = r0 @ r
        beta = (rn / rho) * (alpha / om)
        rho = rn
        p = r + beta * (p - om * v)
    return x, maxit, float(np.linalg.norm(r) / bn)


def run(order, method, iterations, cfl_max, scale, freeze, lin_tol=1e-2, lin_max=60, case_name="plate"):
    import __graft_entry__ as ge
    import port
    cb = ge.load_package()
    case = cb.cases.plate(scale=scale) if case_name == "plate" else cb.cases.sa_plate(scale=scale, mixed=False)
    if order == "first":
        case.cfg.reconstruction = 0
    mesh = cb.HostMesh(case.spec)
    ora = port.PortSolver(mesh, case.cfg, case.bcs)
    n, nv = mesh.n_cells, ora.nv
    rp, cols = ora.structure()
    U = np.asarray(cb.cases.freestream_state(case, n)).reshape(nv, n).copy()

    def resid(Ux):
        ora.set_state(Ux)
        return ora.stages()["res"].reshape(nv, n)

    hist, mx, kry, ref_mon, cfl, fallbacks = [], None, 0, None, 1.0, 0
    t0 = time.time()
    for it in range(1, iterations + 1):
        R = resid(U)
        l2 = np.sqrt((R ** 2).sum(axis=1) / n)
        mon = np.array([l2[0], np.sqrt((l2[1:4] ** 2).sum()), l2[4]] + ([l2[5]] if nv == 6 else []))
        mx = mon if mx is None else np.maximum(mx, mon)
        rel = float((mon / mx).max())
        if not np.isfinite(rel):
            hist.append(["blowup", it])
            break
        if freeze and it == freeze:
            ora.freeze_limiter(True)
        if it <= 50:
            cfl = min(cfl_max, 100.0 ** ((it - 1) / 49))
            if it == 50:
                ref_mon = rel
        elif freeze and it <= freeze:
            cfl = 100.0
            ref_mon = rel
        else:
            cfl = min(cfl_max, 100.0 * max(1.0, ref_mon / rel))
        alpha, vals = ora.jacobian(cfl)
        jfnk = method == "jfnk" and (not freeze or it >= freeze)
        b = -R.T.ravel()
        prec = lambda v: port.sgs_apply(rp, cols, vals, nv, v)  # noqa: E731
        if jfnk:
            # one step length for the whole direction, chosen so that no
            # variable moves by more than 1e-7 of its RMS (the conserved
            # variables differ by orders of magnitude in SI units; rho nu~ is
            # ~1e-5 of rho E)
            su = np.sqrt((U ** 2).mean(axis=1)) + 1e-300
            diag = np.repeat(alpha, nv)

            def op(v):
                w = np.abs(v.reshape(n, nv)).max(axis=0) / su
                if w.max() == 0.0:
                    return np.zeros_like(v)
                eps = 1e-7 / w.max()
                return diag * v + (resid(U + eps * v.reshape(n, nv).T) - R).T.ravel() / eps
            du, k, red = bicgstab(op, prec, b, lin_tol, lin_max)
            if not red < 1.0:  # the linear solve did not reduce: take the Picard step instead
                opp = lambda v: port.bsr_spmv(rp, cols, vals, nv, v)  # noqa: E731
                du, k2, red = bicgstab(opp, prec, b, 1e-3, 30)
                k += k2
                fallbacks += 1
        else:
            op = lambda v: port.bsr_spmv(rp, cols, vals, nv, v)  # noqa: E731
            du, k, red = bicgstab(op, prec, b, 1e-3, 30)
        kry += k
        dU = du.reshape(n, nv).T
        if jfnk:  # relax the step to change density and energy by at most 20%; rho nu~ stays >= 0
            worst = max(np.abs(dU[0] / U[0]).max(), np.abs(dU[4] / U[4]).max())
            if nv == 6:
                floor = 1e-3 * np.sqrt((U[5] ** 2).mean())
                worst = max(worst, np.abs(dU[5] / (np.abs(U[5]) + floor)).max())
            dU = dU * min(1.0, 0.2 / max(worst, 1e-300))
        U = U + dU
        if nv == 6:
            U[5] = np.maximum(U[5], 0.0)
        if it % max(1, iterations // 15) == 0 or rel < 1e-8:
            hist.append([it, float("%.3g" % rel), float("%.3g" % cfl), kry, float("%.2g" % red)])
            kry = 0
        if rel < 1e-8:
            break
    return {"case": case_name, "order": order, "method": method, "cells": n, "cfl_max": cfl_max, "freeze": freeze,
            "wall_s": round(time.time() - t0, 1), "picard_fallbacks": fallbacks, "hist": hist}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", choices=["plate", "sa_plate"], default="plate")
    ap.add_argument("--order", choices=["first", "second"], default="second")
    ap.add_argument("--method", choices=["picard", "jfnk"], default="jfnk")
    ap.add_argument("--iterations", type=int, default=600)
    ap.add_argument("--cfl-max", type=float, default=1000.0)
    ap.add_argument("--scale", type=int, default=8)
    ap.add_argument("--freeze", type=int, default=150)
    a = ap.parse_args()
    print(json.dumps(run(a.order, a.method, a.iterations, a.cfl_max, a.scale, a.freeze, case_name=a.case)))


if __name__ == "__main__":
    main()
