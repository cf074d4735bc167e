"""Runs a case to a 1e-8 residual drop on the reference build, the C
restatement or the GPU library with the same schedule: CFL ramp, limiter
frozen at the end of the ramp, convergence monitor max(mass, |momentum|,
energy) L2 against its running maximum (the library's run_steady)."""
import numpy as np


def monitor(l2):
    l2 = np.asarray(l2)
    return np.array([l2[0], np.sqrt((l2[1:4] ** 2).sum()), l2[4]])


def converge_host(cb, solver, case, U0, max_it=2000, tol=1e-8):
    """Host-driven loop over newton_step of a reference or oracle solver."""
    solver.set_state(U0)
    mx = None
    it = 0
    for it in range(1, max_it + 1):
        if it == case.cfg.limiter_freeze:
            solver.freeze_limiter(True)
        m = monitor(solver.newton_step(cb.cases.cfl_at(case.cfg, it))[:5])
        mx = m if mx is None else np.maximum(mx, m)
        if it > 1 and (m / mx).max() <= tol:
            return solver.get_state(), it
    raise AssertionError(f"no 1e-8 drop in {max_it} iterations")


def field_errors(U, U_ref, gamma=1.4):
    """L2-relative errors of rho, |u| components, p between two conserved
    states (5 x n)."""
    def prim(V):
        rho = V[0]
        u, v, w = V[1] / rho, V[2] / rho, V[3] / rho
        p = (gamma - 1.0) * (V[4] - 0.5 * rho * (u * u + v * v + w * w))
        return {"rho": rho, "u": u, "v": v, "p": p}
    a, b = prim(U), prim(U_ref)
    out = {}
    for k in a:
        scale = np.linalg.norm(b[k])
        if k == "v":  # a cross-flow component: relative to the speed
            scale = np.linalg.norm(np.sqrt(b["u"] ** 2 + b["v"] ** 2))
        out[k] = float(np.linalg.norm(a[k] - b[k]) / max(scale, 1e-300))
    return out
