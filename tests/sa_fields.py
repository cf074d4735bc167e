"""Spalart-Allmaras analytic test fields shared by the CPU (oracle) and GPU
tests: a uniform, unjittered plate mesh with hand-built states for which the
SA-1994 nu_tilde residual has a closed form at interior cells.

Residual convention (as the mean flow): R = sum of outward face fluxes -
V * sources, so that dU/dt = -R / V.  For constant rho and mu:

  R_nu / V = -(1/sigma) div((mu + rho nu) grad nu) - (cb2/sigma) rho |grad nu|^2
             - cb1 Sbar rho nu + cw1 fw rho nu^2 / d^2

with S = sqrt(2 S_ij S_ij) and fw = g ((1 + cw3^6) / (g^6 + cw3^6))^(1/6)
(Spalart & Allmaras 1994; the reference module
include/cfd/solver/compressible/turbulence/spalart_allmaras.hpp adds the
diffusion and cb2 terms with the opposite sign, halves the shear terms of S
and drops cw3^6 from the denominator of fw).
"""
from __future__ import annotations

import numpy as np

SIGMA, CB1, CB2, KAPPA, CW2, CW3, CV1 = 2.0 / 3.0, 0.1355, 0.622, 0.41, 0.3, 2.0, 7.1
CW1 = CB1 / KAPPA ** 2 + (1.0 + CB2) / SIGMA


def uniform_case(cb, wall: bool, nx=40, ny=24, nz=4):
    """SA plate case on a uniform hex mesh (spacing h in x and y, no
    jitter); without `wall` the no-slip patch becomes a symmetry plane so
    that the wall distance is infinite (1e30)."""
    case = cb.cases.sa_plate(scale=8, mixed=False)
    s = case.spec
    s.nx, s.ny, s.nz = nx, ny, nz
    h = s.lx / nx
    s.first_spacing, s.stretch, s.cap_spacing, s.jitter = h, 1.0, 0.0, 0.0
    s.lz = nz * h
    case.cfg.sgs_ordering = cb.SGS_LEVEL
    if not wall:
        case.bcs[3] = cb.bc(3, cb.BC_SYMMETRY)
    return case, h


def state(case, n, rho, T, u_of_y, nu_of_xy, xc, yc):
    """Conserved U (6 x n) with uniform rho and T, u = u_of_y(y) and
    nu_tilde = nu_of_xy(x, y)."""
    R = 287.052874
    p = rho * R * T
    e = R / 0.4 * T
    u = u_of_y(yc)
    U = np.zeros((6, n))
    U[0] = rho
    U[1] = rho * u
    U[4] = rho * e + 0.5 * rho * u * u
    U[5] = rho * nu_of_xy(xc, yc)
    return U, p


def sutherland(T):
    return 1.716e-5 * (273.15 + 110.4) * (T / 273.15) ** 1.5 / (T + 110.4)


def interior(xc, yc, h, lx, ly, layers=3):
    return (xc > layers * h) & (xc < lx - layers * h) & (yc > layers * h) & (yc < ly - layers * h)


def diffusion_expected(rho, mu, nu0, a, x0, y0, xc, yc):
    """R_nu / V for nu = nu0 + a ((x-x0)^2 + (y-y0)^2) at rest without walls
    (production at the Sbar floor 1e-10, no destruction)."""
    nu = nu0 + a * ((xc - x0) ** 2 + (yc - y0) ** 2)
    g2 = (2 * a * (xc - x0)) ** 2 + (2 * a * (yc - y0)) ** 2
    lap = 4.0 * a
    diff = (mu * lap + rho * g2 + rho * nu * lap) / SIGMA
    return -diff - (CB2 / SIGMA) * rho * g2 - CB1 * 1e-10 * rho * nu


def shear_sources_expected(rho, mu, nu, gamma, d):
    """R_nu / V for u = gamma * y, uniform nu (no diffusion, no cb2 term):
    -P + D with S = |gamma|."""
    d = np.maximum(d, 1e-10)
    chi = nu / (mu / rho)
    fv1 = chi ** 3 / (chi ** 3 + CV1 ** 3)
    fv2 = 1.0 - chi / (1.0 + chi * fv1)
    sbar = np.maximum(abs(gamma) + nu * fv2 / (KAPPA ** 2 * d ** 2), 1e-10)
    r = np.clip(nu / (sbar * KAPPA ** 2 * d ** 2), 0.0, 10.0)
    g = r + CW2 * (r ** 6 - r)
    fw = g * ((1.0 + CW3 ** 6) / (g ** 6 + CW3 ** 6)) ** (1.0 / 6.0)
    return -CB1 * sbar * rho * nu + CW1 * fw * rho * nu ** 2 / d ** 2
