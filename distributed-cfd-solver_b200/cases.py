"""Benchmark workloads: mesh spec + solver configuration + boundary patches.

Each case restates one benchmark configuration of the hot path with seeded
synthetic inputs (the reference ships no meshes or datasets):

  ramp  - Mach 2 Euler flow over a 15 deg compression ramp, 64x32x2 hex
  plate - laminar Navier-Stokes flat plate, M=0.5, Re_L=1e5, 256x128x32 hex,
          wall-normal stretching 1.08 from 1e-5 L, +-10% node jitter
  bump  - transonic Euler bump (M=0.85) on 160x80x80 hex split into 6 tets
  sa_plate - Spalart-Allmaras RANS flat plate, M=0.2, Re_L=5e6, 384x192x56
          hex, wall-normal stretching 1.1 from 1e-6 L, +-5% node jitter

Every case takes a `scale` that divides the cell counts for the parity tests.
Free-stream states follow from (M, T, p) or (M, Re_L, T) with the ideal gas
and Sutherland law of the reference (include/cfd/core/types.hpp:36-50).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

from . import (BC_FARFIELD, BC_NO_SLIP_WALL_HEAT_FLUX, BC_SLIP_WALL, BC_SUBSONIC_INLET, BC_SUBSONIC_OUTLET,
               BC_SUPERSONIC_INLET, BC_SUPERSONIC_OUTLET, BC_SYMMETRY, GRAD_LSQ_NODE, JAC_THIN_LAYER,
               LIM_VENKATAKRISHNAN,
               PC_SGS, PREC_FP64, PREFREEZE_FP64, RECON_MUSCL, SGS_COLOR, MeshSpec, bc, default_config)

GAMMA = 1.4
# run_steady freezes the MUSCL limiter from this iteration on, the last of
# the 50-iteration CFL ramp: the limiter's on/off switching otherwise holds
# the residual at a plateau (1e-3 .. 1e-4).  Switching also amplifies
# round-off: two FP64 codes that differ only in their rounding (the
# reference build and its C restatement) drift apart by 3e-8 after 100
# iterations and 1.5e-6 after 300 on the ramp, and each converges to the
# problem its own frozen limiter defines; frozen at the end of the ramp
# they agree to 5e-11 and converge in 279 iterations instead of 464.
LIMITER_FREEZE = 50
# mixed precision and the learned guess start at the freeze (the iterates
# before it are the FP64 path's): every precision solves one frozen problem
PRE_FREEZE = PREFREEZE_FP64
R_GAS = 287.052874


def sutherland(T: float) -> float:
    return 1.716e-5 * (273.15 + 110.4) * (T / 273.15) ** 1.5 / (T + 110.4)


def sound_speed(T: float) -> float:
    return math.sqrt(GAMMA * R_GAS * T)


@dataclass
class Case:
    name: str
    spec: MeshSpec
    cfg: object
    bcs: list
    iterations: int
    description: str
    extra: dict = field(default_factory=dict)


def _spec(kind, nx, ny, nz, lx, ly, lz, seed, **kw) -> MeshSpec:
    s = MeshSpec()
    s.kind, s.nx, s.ny, s.nz = kind, nx, ny, nz
    s.lx, s.ly, s.lz = lx, ly, lz
    s.seed = seed
    s.permute = 1
    s.reorder_rcm = 1
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def ramp(scale: int = 1, seed: int = 1234, iterations: int = 200) -> Case:
    """Inviscid Mach-2 compression ramp (64x32x2 hex, 4,096 cells)."""
    nx, ny, nz = max(64 // scale, 4), max(32 // scale, 2), 2
    T, p, M = 300.0, 101325.0, 2.0
    u = M * sound_speed(T)
    rho = p / (R_GAS * T)
    lx, ly = 1.0, 0.5
    spec = _spec(0, nx, ny, nz, lx, ly, 2.0 * lx / nx, seed, ramp_angle_deg=15.0, ramp_x=0.25, jitter=0.0)
    cfg = default_config(viscous=0, gradient=GRAD_LSQ_NODE, reconstruction=RECON_MUSCL, limiter=LIM_VENKATAKRISHNAN,
                         venkat_k=0.5, precond=PC_SGS, sgs_ordering=SGS_COLOR, precision=PREC_FP64,
                         lin_rel_tol=1e-3, lin_abs_tol=1e-30, lin_max_iterations=30, cfl=1.0, cfl_max=100.0,
                         cfl_ramp_iterations=50, max_iterations=iterations, residual_tolerance=1e-8, convergence_monitor=1,
                         limiter_freeze=LIMITER_FREEZE, pre_freeze=PRE_FREEZE,
                         init_rho=rho, init_p=p, init_velocity=(u, 0.0, 0.0))
    bcs = [bc(0, BC_SUPERSONIC_INLET, p=p, t=T, velocity=(u, 0.0, 0.0)),
           bc(1, BC_SUPERSONIC_OUTLET), bc(2, BC_SUPERSONIC_OUTLET), bc(3, BC_SLIP_WALL), bc(4, BC_SYMMETRY)]
    return Case("ramp", spec, cfg, bcs, iterations, "Euler M=2 15deg compression ramp, 64x32x2 hex",
                {"mach": M, "T": T, "p": p})


def plate(scale: int = 1, seed: int = 4321, iterations: int = 200, mixed: bool = False,
          jacobian: int = JAC_THIN_LAYER) -> Case:
    """Laminar flat plate, M=0.5, Re_L=1e5 (256x128x32 hex, 1,048,576 cells).
    `jacobian=JAC_REFERENCE` selects the reference's viscous Jacobian (for
    comparisons with the reference build)."""
    nx, ny, nz = max(256 // scale, 8), max(128 // scale, 8), max(32 // scale, 2)
    T, M, Re, L = 288.15, 0.5, 1.0e5, 1.0
    u = M * sound_speed(T)
    mu = sutherland(T)
    rho = Re * mu / (u * L)
    p = rho * R_GAS * T
    first = 1.0e-5 * L * scale
    spec = _spec(1, nx, ny, nz, 1.25 * L, 0.0, 0.1 * L, seed, first_spacing=first, stretch=1.08 ** scale,
                 jitter=0.10, plate_x0=0.25 * L)
    cfg = default_config(viscous=1, gradient=GRAD_LSQ_NODE, reconstruction=RECON_MUSCL, limiter=LIM_VENKATAKRISHNAN,
                         venkat_k=0.5, precond=PC_SGS, sgs_ordering=SGS_COLOR,
                         precision=PREC_FP64 if not mixed else 1, prandtl=0.72, jacobian=jacobian,
                         lin_rel_tol=1e-3, lin_abs_tol=1e-30, lin_max_iterations=30, cfl=1.0, cfl_max=100.0,
                         cfl_ramp_iterations=50, max_iterations=iterations, residual_tolerance=1e-8, convergence_monitor=1,
                         limiter_freeze=LIMITER_FREEZE, pre_freeze=PRE_FREEZE,
                         init_rho=rho, init_p=p, init_velocity=(u, 0.0, 0.0))
    # top boundary: symmetry plane (a Riemann far field there switches between
    # its inflow and outflow branches where v ~ 0 and holds a limit cycle)
    bcs = [bc(0, BC_SUBSONIC_INLET, p=p, t=T, velocity=(u, 0.0, 0.0)),
           bc(1, BC_SUBSONIC_OUTLET, p=p),
           bc(2, BC_SYMMETRY),
           bc(3, BC_NO_SLIP_WALL_HEAT_FLUX, tmp_grad=0.0),
           bc(4, BC_SYMMETRY), bc(5, BC_SYMMETRY)]
    return Case("plate", spec, cfg, bcs, iterations, "laminar NS flat plate M=0.5 Re_L=1e5, 256x128x32 hex",
                {"mach": M, "Re": Re, "T": T, "p": p, "rho": rho, "u": u})


def sa_plate(scale: int = 1, seed: int = 2468, iterations: int = 200, mixed: bool = True, mach: float = 0.2,
             reynolds: float = 5.0e6, spec: MeshSpec | None = None) -> Case:
    """Spalart-Allmaras RANS flat plate, M=0.2, Re_L=5e6, free-stream
    nu_tilde/nu = 3 (384x192x56 hex, 4,128,768 cells); wall-normal growth 1.1
    from 1e-6 L, capped at 0.01 L.  `spec` replaces the mesh (the learned
    guess's training flows run on the laminar plate's mesh)."""
    nx, ny, nz = max(384 // scale, 8), max(192 // scale, 8), max(56 // scale, 2)
    T, M, Re, L = 288.15, mach, reynolds, 1.0
    u = M * sound_speed(T)
    mu = sutherland(T)
    rho = Re * mu / (u * L)
    p = rho * R_GAS * T
    if spec is None:
        spec = _spec(1, nx, ny, nz, 1.25 * L, 0.0, 0.1 * L, seed, first_spacing=1.0e-6 * L * scale,
                     stretch=1.1 ** scale, cap_spacing=0.01 * L * scale, jitter=0.05, plate_x0=0.25 * L)
    cfg = default_config(viscous=1, turbulence=1, nu_inf_ratio=3.0, gradient=GRAD_LSQ_NODE,
                         reconstruction=RECON_MUSCL, limiter=LIM_VENKATAKRISHNAN, venkat_k=0.5, precond=PC_SGS,
                         sgs_ordering=SGS_COLOR, precision=1 if mixed else PREC_FP64, prandtl=0.72,
                         jacobian=JAC_THIN_LAYER,
                         lin_rel_tol=1e-3, lin_abs_tol=1e-30, lin_max_iterations=30, cfl=1.0, cfl_max=100.0,
                         cfl_ramp_iterations=50, max_iterations=iterations, residual_tolerance=1e-8, convergence_monitor=1,
                         limiter_freeze=LIMITER_FREEZE, pre_freeze=PRE_FREEZE,
                         init_rho=rho, init_p=p, init_velocity=(u, 0.0, 0.0))
    bcs = [bc(0, BC_SUBSONIC_INLET, p=p, t=T, velocity=(u, 0.0, 0.0)),
           bc(1, BC_SUBSONIC_OUTLET, p=p),
           bc(2, BC_SYMMETRY),
           bc(3, BC_NO_SLIP_WALL_HEAT_FLUX, tmp_grad=0.0),
           bc(4, BC_SYMMETRY), bc(5, BC_SYMMETRY)]
    return Case("sa_plate", spec, cfg, bcs, iterations, "SA RANS flat plate M=0.2 Re_L=5e6, 384x192x56 hex",
                {"mach": M, "Re": Re, "T": T, "p": p, "rho": rho, "u": u, "nu_inf": 3.0 * mu / rho})


def sa_training_flows(scale: int = 4, iterations: int = 200) -> list[Case]:
    """The learned guess's training flows for the SA plate: Spalart-Allmaras
    on the laminar plate's mesh (256x128x32 hex divided by `scale` per
    direction, wall spacing 1e-5 L, growth 1.08) at M in {0.15, 0.2, 0.3} and
    Re_L in {1e6, 5e6, 1e7}, mixed precision.  The compression ramp's
    supersonic Euler block has no wall for the turbulence model and is not
    used."""
    spec = plate(scale=scale).spec
    return [sa_plate(iterations=iterations, mixed=True, mach=m, reynolds=re, spec=spec)
            for m in (0.15, 0.2, 0.3) for re in (1.0e6, 5.0e6, 1.0e7)]


def bump(scale: int = 1, seed: int = 777, iterations: int = 200, mixed: bool = True, mach: float = 0.85) -> Case:
    """Transonic Euler bump, M=0.85, 160x80x80 hex -> 6 tets each (6,144,000 cells).
    CFL 1 -> 50 (at 100 the transient near the end of the ramp is marginal:
    round-off differences decide whether it survives)."""
    nx, ny, nz = max(160 // scale, 6), max(80 // scale, 3), max(80 // scale, 3)
    T, p, M = 288.15, 101325.0, mach
    u = M * sound_speed(T)
    rho = p / (R_GAS * T)
    spec = _spec(2, nx, ny, nz, 3.0, 1.5, 1.5, seed, bump_height=0.1, bump_x0=1.0, bump_x1=2.0, jitter=0.05)
    cfg = default_config(viscous=0, gradient=GRAD_LSQ_NODE, reconstruction=RECON_MUSCL, limiter=LIM_VENKATAKRISHNAN,
                         venkat_k=0.5, precond=PC_SGS, sgs_ordering=SGS_COLOR,
                         precision=1 if mixed else PREC_FP64,
                         lin_rel_tol=1e-3, lin_abs_tol=1e-30, lin_max_iterations=30, cfl=1.0, cfl_max=50.0,
                         cfl_ramp_iterations=50, max_iterations=iterations, residual_tolerance=1e-8, convergence_monitor=1,
                         limiter_freeze=LIMITER_FREEZE, pre_freeze=PRE_FREEZE,
                         init_rho=rho, init_p=p, init_velocity=(u, 0.0, 0.0))
    far = dict(p=p, t=T, velocity=(u, 0.0, 0.0))
    bcs = [bc(0, BC_FARFIELD, **far), bc(1, BC_FARFIELD, **far), bc(2, BC_FARFIELD, **far), bc(3, BC_SLIP_WALL),
           bc(4, BC_SYMMETRY)]
    return Case("bump", spec, cfg, bcs, iterations, "transonic Euler bump M=0.85, 160x80x80x6 tets",
                {"mach": M, "T": T, "p": p})


def cfl_at(cfg, it: int) -> float:
    """CFL of nonlinear iteration `it` (1-based): geometric ramp from cfg.cfl
    to cfg.cfl_max over cfg.cfl_ramp_iterations (the library's run_steady
    schedule)."""
    K = cfg.cfl_ramp_iterations
    if K <= 1 or not cfg.cfl_max > cfg.cfl:
        return cfg.cfl
    t = min(1.0, (it - 1) / (K - 1))
    return min(cfg.cfl_max, cfg.cfl * (cfg.cfl_max / cfg.cfl) ** t)


def freestream_state(case: Case, n: int):
    """Conserved state U (5 x n, 6 x n with Spalart-Allmaras) of the case's
    uniform initial condition."""
    import numpy as np
    cfg = case.cfg
    rho, p = cfg.init_rho, cfg.init_p
    u, v, w = cfg.init_velocity[0], cfg.init_velocity[1], cfg.init_velocity[2]
    T = p / (rho * R_GAS)
    e = R_GAS / (GAMMA - 1.0) * T
    sa = bool(cfg.turbulence)
    U = np.empty((6 if sa else 5, n))
    U[0], U[1], U[2], U[3] = rho, rho * u, rho * v, rho * w
    U[4] = rho * e + 0.5 * rho * (u * u + v * v + w * w)
    if sa:
        U[5] = cfg.nu_inf_ratio * sutherland(T) / rho * rho
    return U


def perturbed_state(case: Case, n: int, seed: int = 5, amplitude: float = 0.02):
    """Free stream with a smooth seeded perturbation (non-trivial gradients,
    active limiter) for the stage-by-stage parity tests."""
    import numpy as np
    rng = np.random.default_rng(seed)
    U = freestream_state(case, n)
    base = U.copy()
    for k in range(U.shape[0]):
        U[k] = base[k] * (1.0 + amplitude * rng.uniform(-1.0, 1.0, size=n))
    # keep the velocity perturbation relative to the free-stream speed
    spd = max(abs(case.cfg.init_velocity[0]), 1.0) * base[0]
    U[2] = base[2] + amplitude * spd * rng.uniform(-1, 1, size=n)
    U[3] = base[3] + amplitude * spd * rng.uniform(-1, 1, size=n)
    return U
