"""Python host mirror of the B200 hot-path library (include/cfdg.h).

The product is the C-ABI shared library ``libcfdg.so`` built next to this
file (hand-written sm_100a CUDA behind a C++ host).  This module binds it
with ctypes and mirrors the reference solver's entry points for the path:

  Solver.evaluate_residual   Solver::evaluate_residual   (solver.hpp:169-247)
  Solver.compute_dt          Solver::compute_dt          (solver.hpp:256-287)
  Solver.assemble_jacobian   Solver::assemble_jacobian   (solver.hpp:249-254)
  Solver.linear_solve        BSRLinearSystem::solve      (bsr_linear_system.hpp:93-97)
  Solver.newton_step         BackwardEuler::advance      (implicit_euler.hpp:34-76)
  Solver.run_steady          Solver::run_steady          (solver.hpp:597-660)
  Bsr.spmv / sgs_* / bicgstab  BsrMatrix::apply, SgsPreconditioner, BiCGSTAB::solve

Errors are raised as CfdgError carrying the library status and message; a
missing library raises immediately (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libcfdg.so"

# ------------------------------------------------------------------ constants
OK = 0
ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_SINGULAR, ERR_NONFINITE = -1, -2, -3, -4, -5
ERR_DIVERGED, ERR_MESH, ERR_UNSUPPORTED, ERR_NODEVICE = -6, -7, -8, -9

TET, PYRA, PRISM, HEXA, TRI, QUAD = range(6)
(BC_SUPERSONIC_INLET, BC_SUPERSONIC_OUTLET, BC_SUBSONIC_INLET, BC_SUBSONIC_OUTLET, BC_SLIP_WALL,
 BC_NO_SLIP_WALL, BC_NO_SLIP_WALL_HEAT_FLUX, BC_SYMMETRY, BC_FARFIELD) = range(9)
INFLOW_VELOCITY, INFLOW_MACH_ANGLES, INFLOW_MACH_DIRECTION = range(3)
GRAD_LSQ_FACE, GRAD_LSQ_NODE = 2, 3
RECON_FIRST_ORDER, RECON_MUSCL = 0, 1
LIM_VENKATAKRISHNAN, LIM_BARTH_JESPERSEN, LIM_VAN_ALBADA = 1, 2, 3
SGS_LEVEL, SGS_COLOR = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
PC_NONE, PC_SGS = 0, 1
KRYLOV_CONVERGED, KRYLOV_DIVERGED, KRYLOV_MAX_ITERATIONS = 0, 1, 2
(FIELD_U, FIELD_Q, FIELD_GRAD, FIELD_PHI, FIELD_RES, FIELD_LAM, FIELD_DT, FIELD_ALPHA, FIELD_JAC, FIELD_DU,
 FIELD_MUT, FIELD_WALLDIST, FIELD_RHS, FIELD_NU, FIELD_NU_GRAD) = range(15)
JAC_REFERENCE, JAC_THIN_LAYER = 0, 1
KRYLOV_DEVICE_LOOP, KRYLOV_HOST_LOOP = 0, 1
PREFREEZE_CONFIGURED, PREFREEZE_FP64 = 0, 1
TIME_STEADY, TIME_UNSTEADY = 0, 1
NEWTON_PICARD, NEWTON_JACOBIAN_FREE = 0, 1
# cfdg_halo_get arrays (CFDG_HALO_*)
CFDG_HALO_ARRAYS = {"local_to_global": 0, "nb_ranks": 1, "send_offsets": 2, "send_owned_local": 3,
                    "recv_offsets": 4, "recv_ghost_local": 5}
JF_BICGSTAB, JF_GMRES = 0, 1
STAGE_PRIMITIVES, STAGE_GRADIENT, STAGE_LIMITER, STAGE_FLUXES = range(4)
KCAT_NAMES = ("primitives", "gradient", "limiter", "face_flux", "cell_gather", "jacobian", "lu", "spmv", "sgs",
              "krylov", "update", "turbulence", "guess", "jfnk")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_fp = C.POINTER(C.c_float)
_u16p = C.POINTER(C.c_uint16)
MLP_IN, MLP_HID, MLP_OUT = 48, 64, 16
_up = C.POINTER(C.c_uint8)


class MeshHost(C.Structure):
    _fields_ = [("n_cells", C.c_int32), ("n_faces", C.c_int32), ("n_inner_faces", C.c_int32),
                ("n_nodes", C.c_int32), ("n_patches", C.c_int32),
                ("cell_type", _up), ("cell_nodes_offsets", _ip), ("cell_nodes", _ip),
                ("node_x", _dp), ("node_y", _dp), ("node_z", _dp),
                ("cell_centroid_x", _dp), ("cell_centroid_y", _dp), ("cell_centroid_z", _dp), ("cell_volume", _dp),
                ("face_owner", _ip), ("face_neigh", _ip), ("face_patch", _ip),
                ("face_nodes_offsets", _ip), ("face_nodes", _ip),
                ("face_centroid_x", _dp), ("face_centroid_y", _dp), ("face_centroid_z", _dp),
                ("face_normal_x", _dp), ("face_normal_y", _dp), ("face_normal_z", _dp), ("face_area", _dp)]


class BcDesc(C.Structure):
    _fields_ = [("patch_id", C.c_int32), ("type", C.c_int32), ("inflow_mode", C.c_int32), ("pad_", C.c_int32),
                ("p", C.c_double), ("t", C.c_double), ("tmp_grad", C.c_double), ("velocity", C.c_double * 3),
                ("mach", C.c_double), ("alpha_deg", C.c_double), ("beta_deg", C.c_double),
                ("direction", C.c_double * 3)]


class Config(C.Structure):
    _fields_ = [("viscous", C.c_int32), ("turbulence", C.c_int32), ("gradient", C.c_int32),
                ("reconstruction", C.c_int32), ("limiter", C.c_int32), ("precision", C.c_int32),
                ("precond", C.c_int32), ("sgs_ordering", C.c_int32), ("sgs_sweeps", C.c_int32),
                ("lin_max_iterations", C.c_int32), ("cfl_ramp_iterations", C.c_int32),
                ("residual_interval", C.c_int32), ("convergence_monitor", C.c_int32), ("jacobian", C.c_int32),
                ("limiter_freeze", C.c_int32), ("krylov_loop", C.c_int32), ("pre_freeze", C.c_int32),
                ("reserved_", C.c_int32),
                ("gamma", C.c_double), ("gas_constant", C.c_double), ("prandtl", C.c_double),
                ("prandtl_turb", C.c_double), ("init_rho", C.c_double), ("init_p", C.c_double),
                ("init_velocity", C.c_double * 3), ("venkat_k", C.c_double), ("cfl", C.c_double),
                ("cfl_max", C.c_double), ("residual_tolerance", C.c_double), ("lin_rel_tol", C.c_double),
                ("lin_abs_tol", C.c_double), ("nu_inf_ratio", C.c_double), ("max_iterations", C.c_int64),
                ("dt_physical", C.c_double), ("max_time_steps", C.c_int64), ("time_mode", C.c_int32),
                ("bdf_order", C.c_int32), ("newton_operator", C.c_int32), ("jf_max_iterations", C.c_int32),
                ("jf_rel_tol", C.c_double), ("jf_eps", C.c_double), ("jf_max_change", C.c_double),
                ("cfl_ser_max", C.c_double), ("jf_krylov", C.c_int32), ("jf_restart", C.c_int32),
                ("jf_accept", C.c_double)]


class UnsteadyResult(C.Structure):
    _fields_ = [("time_steps", C.c_int64), ("subiterations_total", C.c_int64), ("krylov_iterations_total", C.c_int64),
                ("steps_converged", C.c_int32), ("blowup", C.c_int32), ("t_physical", C.c_double),
                ("seconds", C.c_double), ("l2_last", C.c_double * 6)]


class KrylovResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int32), ("initial_residual", C.c_double),
                ("final_residual", C.c_double)]


class StepResult(C.Structure):
    _fields_ = [("l2", C.c_double * 6), ("cfl", C.c_double), ("nvars", C.c_int32), ("krylov_status", C.c_int32),
                ("krylov_iterations", C.c_int32), ("guess_used", C.c_int32), ("krylov_initial", C.c_double),
                ("krylov_final", C.c_double), ("krylov_rhs", C.c_double), ("jacobian_free", C.c_int32),
                ("picard_fallback", C.c_int32), ("step_scale", C.c_double)]


class RunResult(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("converged", C.c_int32), ("blowup", C.c_int32), ("rel", C.c_double),
                ("seconds", C.c_double), ("krylov_iterations_total", C.c_int64), ("l2_first", C.c_double * 6),
                ("l2_last", C.c_double * 6), ("jacobian_free_steps", C.c_int64), ("picard_fallbacks", C.c_int64),
                ("cfl_last", C.c_double)]


class MeshSpec(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double), ("first_spacing", C.c_double),
                ("stretch", C.c_double), ("cap_spacing", C.c_double), ("jitter", C.c_double),
                ("ramp_angle_deg", C.c_double), ("ramp_x", C.c_double), ("plate_x0", C.c_double),
                ("bump_height", C.c_double), ("bump_x0", C.c_double), ("bump_x1", C.c_double),
                ("seed", C.c_uint64), ("permute", C.c_int32), ("reorder_rcm", C.c_int32)]


class CfdgError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"cfdg status {status}: {message}")
        self.status = status


_LIB = None

# Exported symbols and their ctypes signatures (also the symbol list the
# CPU-side tests check against include/cfdg.h).
_SIGS = {
    "cfdg_version": (C.c_int, []),
    "cfdg_status_string": (C.c_char_p, [C.c_int]),
    "cfdg_last_error": (C.c_char_p, []),
    "cfdg_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "cfdg_config_default": (None, [C.POINTER(Config)]),
    "cfdg_mesh_generate": (C.c_int, [C.POINTER(MeshSpec), C.POINTER(C.c_void_p)]),
    "cfdg_host_mesh_view": (C.c_int, [C.c_void_p, C.POINTER(MeshHost)]),
    "cfdg_host_mesh_free": (C.c_int, [C.c_void_p]),
    "cfdg_mesh_compute_geometry": (C.c_int, [C.c_void_p]),
    "cfdg_solver_create": (C.c_int, [C.c_int, C.POINTER(MeshHost), C.POINTER(Config), C.POINTER(BcDesc), C.c_int32,
                                     C.POINTER(C.c_void_p)]),
    "cfdg_solver_destroy": (C.c_int, [C.c_void_p]),
    "cfdg_solver_init_fields": (C.c_int, [C.c_void_p]),
    "cfdg_solver_set_state": (C.c_int, [C.c_void_p, _dp, C.c_int64]),
    "cfdg_solver_get_field": (C.c_int, [C.c_void_p, C.c_int32, _dp, C.c_int64]),
    "cfdg_solver_sizes": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "cfdg_evaluate_residual": (C.c_int, [C.c_void_p]),
    "cfdg_solver_stage": (C.c_int, [C.c_void_p, C.c_int32]),
    "cfdg_compute_dt": (C.c_int, [C.c_void_p, C.c_double]),
    "cfdg_assemble_jacobian": (C.c_int, [C.c_void_p]),
    "cfdg_linear_solve": (C.c_int, [C.c_void_p, C.POINTER(KrylovResult)]),
    "cfdg_newton_step": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(StepResult)]),
    "cfdg_residual_norms": (C.c_int, [C.c_void_p, _dp]),
    "cfdg_run_steady": (C.c_int, [C.c_void_p, C.POINTER(RunResult)]),
    "cfdg_run_unsteady": (C.c_int, [C.c_void_p, C.POINTER(UnsteadyResult)]),
    "cfdg_solver_reset_time_levels": (C.c_int, [C.c_void_p]),
    "cfdg_solver_write_vtu": (C.c_int, [C.c_void_p, C.POINTER(MeshHost), C.c_char_p, C.c_char_p]),
    "cfdg_solver_freeze_limiter": (C.c_int, [C.c_void_p, C.c_int32]),
    "cfdg_solver_set_limiter": (C.c_int, [C.c_void_p, _dp, C.c_int64]),
    "cfdg_tc_selftest": (C.c_int, [C.c_int, C.c_int32, C.c_int32, _u16p, _u16p, _fp]),
    "cfdg_mlp_create": (C.c_int, [C.c_int, C.c_int32, C.c_uint64, C.POINTER(C.c_void_p)]),
    "cfdg_mlp_destroy": (C.c_int, [C.c_void_p]),
    "cfdg_mlp_param_count": (C.c_int32, []),
    "cfdg_mlp_get_params": (C.c_int, [C.c_void_p, _fp, C.c_int64]),
    "cfdg_mlp_set_params": (C.c_int, [C.c_void_p, _fp, C.c_int64]),
    "cfdg_mlp_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "cfdg_mlp_forward_host": (C.c_int, [C.c_void_p, _u16p, C.c_int64, _dp]),
    "cfdg_mlp_gradient_host": (C.c_int, [C.c_void_p, _u16p, _fp, C.c_int64, _fp, _fp]),
    "cfdg_mlp_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_float, C.c_uint64, _fp]),
    "cfdg_dataset_create": (C.c_int, [C.c_int, C.c_int32, C.c_int64, C.POINTER(C.c_void_p)]),
    "cfdg_dataset_destroy": (C.c_int, [C.c_void_p]),
    "cfdg_dataset_size": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "cfdg_dataset_clear": (C.c_int, [C.c_void_p]),
    "cfdg_dataset_append_host": (C.c_int, [C.c_void_p, _u16p, _fp, C.c_int64]),
    "cfdg_dataset_read_host": (C.c_int, [C.c_void_p, _u16p, _fp, C.c_int64]),
    "cfdg_solver_attach_guess": (C.c_int, [C.c_void_p, C.c_void_p]),
    "cfdg_solver_attach_dataset": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int32]),
    "cfdg_residual_norms_noalloc": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, _dp]),
    "cfdg_solver_stream": (C.c_void_p, [C.c_void_p]),
    "cfdg_solver_launch_count": (C.c_int64, [C.c_void_p]),
    "cfdg_solver_profile": (C.c_int, [C.c_void_p, C.c_int32]),
    "cfdg_solver_profile_read": (C.c_int, [C.c_void_p, _dp, C.POINTER(C.c_int64), _dp]),
    "cfdg_solver_sgs_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "cfdg_recon_create": (C.c_int, [C.c_int, C.POINTER(MeshHost), C.c_int32, C.c_int32, C.c_double,
                                    C.POINTER(C.c_void_p)]),
    "cfdg_recon_destroy": (C.c_int, [C.c_void_p]),
    "cfdg_gradient": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                C.POINTER(C.c_void_p), C.c_int32, C.c_void_p]),
    "cfdg_limiter": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                               C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int32, C.c_void_p]),
    "cfdg_halo_create": (C.c_int, [C.POINTER(MeshHost), C.c_int32, _ip, C.c_int32, C.POINTER(C.c_void_p)]),
    "cfdg_halo_destroy": (C.c_int, [C.c_void_p]),
    "cfdg_halo_sizes": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "cfdg_halo_get": (C.c_int, [C.c_void_p, C.c_int32, _ip, C.c_int64]),
    "cfdg_halo_pack": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.c_int32, C.c_void_p, C.c_void_p]),
    "cfdg_halo_unpack": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int32, C.POINTER(C.c_void_p), C.c_void_p]),
    "cfdg_halo_pack_blocks": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "cfdg_halo_unpack_blocks": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p]),
    "cfdg_bsr_create": (C.c_int, [C.c_int, C.c_int32, C.c_int32, _ip, _ip, C.c_int32, C.POINTER(C.c_void_p)]),
    "cfdg_bsr_destroy": (C.c_int, [C.c_void_p]),
    "cfdg_bsr_set_values": (C.c_int, [C.c_void_p, _dp]),
    "cfdg_bsr_spmv": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double]),
    "cfdg_bsr_spmv_host": (C.c_int, [C.c_void_p, _dp, _dp, C.c_double, C.c_double]),
    "cfdg_sgs_setup": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "cfdg_sgs_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "cfdg_sgs_apply_host": (C.c_int, [C.c_void_p, _dp, _dp]),
    "cfdg_bicgstab": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_void_p, C.c_void_p,
                                C.POINTER(KrylovResult)]),
    "cfdg_bicgstab_host": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.c_double, C.c_int32, _dp, _dp,
                                     C.POINTER(KrylovResult)]),
    "cfdg_gmres": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_int32, C.c_void_p,
                             C.c_void_p, C.POINTER(KrylovResult)]),
    "cfdg_gmres_host": (C.c_int, [C.c_void_p, C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_int32, _dp, _dp,
                                  C.POINTER(KrylovResult)]),
}


def lib():
    """Loads libcfdg.so (raises if it was not built: no fallback path exists)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with python {PKG_DIR / 'build.py'}")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(status: int) -> None:
    if status != OK:
        msg = lib().cfdg_last_error()
        raise CfdgError(status, msg.decode() if msg else "")


def device_count() -> int:
    n = C.c_int(0)
    check(lib().cfdg_device_count(C.byref(n)))
    return n.value


# cfdg_config_default's values (SolverConfig / SolverParams defaults of the
# reference, include/cfd/solver/compressible/config.hpp:94-136 and
# linalg/config.hpp:14-26), kept here so that configurations can be written
# without loading the library (tests/test_abi_cpu.py checks the two agree).
CONFIG_DEFAULTS = dict(
    viscous=0, turbulence=0, gradient=GRAD_LSQ_NODE, reconstruction=RECON_MUSCL, limiter=LIM_VENKATAKRISHNAN,
    precision=PREC_FP64, precond=PC_SGS, sgs_ordering=SGS_COLOR, sgs_sweeps=1, lin_max_iterations=500,
    cfl_ramp_iterations=0, residual_interval=1, convergence_monitor=0, jacobian=JAC_REFERENCE, limiter_freeze=0,
    krylov_loop=KRYLOV_DEVICE_LOOP, pre_freeze=PREFREEZE_CONFIGURED, reserved_=0,
    gamma=1.4, gas_constant=287.052874, prandtl=0.71, prandtl_turb=0.9, init_rho=1.225, init_p=101325.0,
    init_velocity=(0.0, 0.0, 0.0), venkat_k=0.5, cfl=0.4, cfl_max=0.4, residual_tolerance=1.0e-10,
    lin_rel_tol=1.0e-1, lin_abs_tol=1.0e-15, nu_inf_ratio=3.0, max_iterations=10000,
    dt_physical=1.0e-6, max_time_steps=1, time_mode=TIME_STEADY, bdf_order=2,
    newton_operator=NEWTON_PICARD, jf_max_iterations=60, jf_rel_tol=1.0e-2, jf_eps=1.0e-7, jf_max_change=0.2,
    cfl_ser_max=0.0, jf_krylov=JF_GMRES, jf_restart=30, jf_accept=0.5)


def default_config(**overrides) -> Config:
    cfg = Config()
    for k, v in {**CONFIG_DEFAULTS, **overrides}.items():
        if k == "init_velocity":
            for i in range(3):
                cfg.init_velocity[i] = v[i]
        else:
            setattr(cfg, k, v)
    return cfg


def bc(patch_id: int, kind: int, **kw) -> BcDesc:
    d = BcDesc()
    d.patch_id, d.type = patch_id, kind
    d.inflow_mode = kw.pop("inflow_mode", INFLOW_VELOCITY)
    d.p = kw.pop("p", 101325.0)
    d.t = kw.pop("t", 288.15)
    d.tmp_grad = kw.pop("tmp_grad", 0.0)
    vel = kw.pop("velocity", (0.0, 0.0, 0.0))
    dirn = kw.pop("direction", (1.0, 0.0, 0.0))
    for i in range(3):
        d.velocity[i] = vel[i]
        d.direction[i] = dirn[i]
    d.mach = kw.pop("mach", 0.0)
    d.alpha_deg = kw.pop("alpha_deg", 0.0)
    d.beta_deg = kw.pop("beta_deg", 0.0)
    if kw:
        raise TypeError(f"unknown BC parameters {sorted(kw)}")
    return d


def _np(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


class HostMesh:
    """A synthetic single-partition mesh (cfdg_mesh_generate)."""

    def __init__(self, spec: MeshSpec):
        h = C.c_void_p()
        check(lib().cfdg_mesh_generate(C.byref(spec), C.byref(h)))
        self._h = h
        self.spec = spec
        self.view = MeshHost()
        check(lib().cfdg_host_mesh_view(self._h, C.byref(self.view)))

    def close(self):
        if getattr(self, "_h", None):
            lib().cfdg_host_mesh_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def n_cells(self) -> int:
        return self.view.n_cells

    @property
    def n_faces(self) -> int:
        return self.view.n_faces

    @property
    def n_inner(self) -> int:
        return self.view.n_inner_faces

    def arrays(self) -> dict:
        v = self.view
        n, nf, nn = v.n_cells, v.n_faces, v.n_nodes
        ncn = int(np.ctypeslib.as_array(v.cell_nodes_offsets, shape=(n + 1,))[n])
        nfn = int(np.ctypeslib.as_array(v.face_nodes_offsets, shape=(nf + 1,))[nf])
        out = {
            "cell_type": _np(v.cell_type, n, np.uint8),
            "cell_nodes_offsets": _np(v.cell_nodes_offsets, n + 1, np.int32),
            "cell_nodes": _np(v.cell_nodes, ncn, np.int32),
            "face_nodes_offsets": _np(v.face_nodes_offsets, nf + 1, np.int32),
            "face_nodes": _np(v.face_nodes, nfn, np.int32),
        }
        for k in ("node_x", "node_y", "node_z"):
            out[k] = _np(getattr(v, k), nn, np.float64)
        for k in ("cell_centroid_x", "cell_centroid_y", "cell_centroid_z", "cell_volume"):
            out[k] = _np(getattr(v, k), n, np.float64)
        for k in ("face_owner", "face_neigh", "face_patch"):
            out[k] = _np(getattr(v, k), nf, np.int32)
        for k in ("face_centroid_x", "face_centroid_y", "face_centroid_z", "face_normal_x", "face_normal_y",
                  "face_normal_z", "face_area"):
            out[k] = _np(getattr(v, k), nf, np.float64)
        return out


def _dptr_int(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class Solver:
    """cfdg_solver: the device-resident compressible solver for one mesh."""

    def __init__(self, mesh: HostMesh, cfg: Config, bcs, device: int = 0):
        self.mesh = mesh
        self.cfg = cfg
        arr = (BcDesc * len(bcs))(*bcs)
        h = C.c_void_p()
        check(lib().cfdg_solver_create(device, C.byref(mesh.view), C.byref(cfg), arr, len(bcs), C.byref(h)))
        self._h = h
        sz = (C.c_int64 * 7)()
        check(lib().cfdg_solver_sizes(self._h, sz))
        self.n_cells, self.n_faces, self.n_inner, self.n_total, self.nnzb, self.bs, self.nvars = [int(x) for x in sz]

    def close(self):
        if getattr(self, "_h", None):
            lib().cfdg_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def init_fields(self):
        check(lib().cfdg_solver_init_fields(self._h))

    def set_state(self, U: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.nvars, -1)
        check(lib().cfdg_solver_set_state(self._h, _dptr(U), U.shape[1]))

    def field_size(self, field: int) -> int:
        n, nt = self.n_cells, self.n_total
        return {FIELD_U: n * self.nvars, FIELD_Q: nt * 5, FIELD_GRAD: nt * 3 * self.nvars, FIELD_PHI: n * 5,
                FIELD_RES: n * self.nvars, FIELD_LAM: n, FIELD_DT: n, FIELD_ALPHA: n,
                FIELD_JAC: self.nnzb * self.bs * self.bs, FIELD_DU: n * self.nvars, FIELD_MUT: nt,
                FIELD_WALLDIST: n, FIELD_RHS: n * self.nvars, FIELD_NU: n, FIELD_NU_GRAD: 3 * nt}[field]

    def get(self, field: int) -> np.ndarray:
        try:
            size = self.field_size(field)
        except KeyError:
            size = 1  # unknown field id: let the library report it
        out = np.empty(size, dtype=np.float64)
        check(lib().cfdg_solver_get_field(self._h, field, _dptr(out), out.size))
        return out

    def stage(self, st: int):
        check(lib().cfdg_solver_stage(self._h, st))

    def evaluate_residual(self):
        check(lib().cfdg_evaluate_residual(self._h))

    def compute_dt(self, cfl: float):
        check(lib().cfdg_compute_dt(self._h, cfl))

    def assemble_jacobian(self):
        check(lib().cfdg_assemble_jacobian(self._h))

    def linear_solve(self) -> KrylovResult:
        r = KrylovResult()
        check(lib().cfdg_linear_solve(self._h, C.byref(r)))
        return r

    def newton_step(self, cfl: float) -> StepResult:
        r = StepResult()
        check(lib().cfdg_newton_step(self._h, cfl, C.byref(r)))
        return r

    def residual_norms(self) -> np.ndarray:
        out = np.zeros(6)
        check(lib().cfdg_residual_norms(self._h, _dptr(out)))
        return out[: self.nvars]

    def attach_guess(self, mlp: "Mlp | None"):
        check(lib().cfdg_solver_attach_guess(self._h, mlp._h if mlp is not None else None))

    def attach_dataset(self, ds: "Dataset | None", stride: int = 1):
        check(lib().cfdg_solver_attach_dataset(self._h, ds._h if ds is not None else None, stride))

    def set_limiter(self, phi):
        """Loads limiter values (5 x n) and freezes them."""
        phi = np.ascontiguousarray(phi, dtype=np.float64).ravel()
        check(lib().cfdg_solver_set_limiter(self._h, _dptr(phi), phi.size))

    def freeze_limiter(self, frozen: bool = True):
        check(lib().cfdg_solver_freeze_limiter(self._h, 1 if frozen else 0))

    def run_steady(self) -> RunResult:
        r = RunResult()
        check(lib().cfdg_run_steady(self._h, C.byref(r)))
        return r

    def run_unsteady(self) -> UnsteadyResult:
        r = UnsteadyResult()
        check(lib().cfdg_run_unsteady(self._h, C.byref(r)))
        return r

    def reset_time_levels(self):
        check(lib().cfdg_solver_reset_time_levels(self._h))

    def write_vtu(self, outdir: str, stem: str):
        """<outdir>/<stem>_00000.vtu + <stem>.pvtu of the current state."""
        check(lib().cfdg_solver_write_vtu(self._h, C.byref(self.mesh.view), str(outdir).encode(), stem.encode()))

    def stream(self) -> int:
        return lib().cfdg_solver_stream(self._h) or 0

    def launch_count(self) -> int:
        return int(lib().cfdg_solver_launch_count(self._h))

    def profile(self, enable: bool):
        check(lib().cfdg_solver_profile(self._h, 1 if enable else 0))

    def profile_read(self) -> dict:
        ms = np.zeros(len(KCAT_NAMES))
        by = np.zeros(len(KCAT_NAMES))
        cnt = (C.c_int64 * len(KCAT_NAMES))()
        check(lib().cfdg_solver_profile_read(self._h, _dptr(ms), cnt, _dptr(by)))
        return {name: {"ms": float(ms[i]), "launches": int(cnt[i]), "bytes": float(by[i])}
                for i, name in enumerate(KCAT_NAMES)}

    def sgs_groups(self):
        f, b = C.c_int32(), C.c_int32()
        check(lib().cfdg_solver_sgs_info(self._h, C.byref(f), C.byref(b)))
        return f.value, b.value


def _u16(a: np.ndarray):
    return a.ctypes.data_as(_u16p)


def _f32(a: np.ndarray):
    return a.ctypes.data_as(_fp)


def to_bf16_bits(x) -> np.ndarray:
    """float array -> bf16 bit patterns (round to nearest even)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def from_bf16_bits(b) -> np.ndarray:
    return (np.ascontiguousarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def tc_selftest(a_bits: np.ndarray, b_bits: np.ndarray, device: int = 0) -> np.ndarray:
    """D[128 x n] = A[128 x k] B[n x k]^T on the tcgen05 tensor cores."""
    a = np.ascontiguousarray(a_bits, dtype=np.uint16)
    b = np.ascontiguousarray(b_bits, dtype=np.uint16)
    n, k = b.shape
    d = np.zeros((128, n), dtype=np.float32)
    check(lib().cfdg_tc_selftest(device, n, k, _u16(a), _u16(b), _f32(d)))
    return d


class Mlp:
    """cfdg_mlp: the learned initial-guess network (device resident)."""

    def __init__(self, nvars: int, seed: int = 1, device: int = 0):
        h = C.c_void_p()
        check(lib().cfdg_mlp_create(device, nvars, seed, C.byref(h)))
        self._h = h
        self.nvars = nvars

    def close(self):
        if getattr(self, "_h", None):
            lib().cfdg_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def param_count() -> int:
        return int(lib().cfdg_mlp_param_count())

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.param_count(), dtype=np.float32)
        check(lib().cfdg_mlp_get_params(self._h, _f32(p), p.size))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib().cfdg_mlp_set_params(self._h, _f32(p), p.size))

    def forward(self, feat_bits: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(feat_bits, dtype=np.uint16).reshape(-1, MLP_IN)
        out = np.zeros((f.shape[0], self.nvars))
        check(lib().cfdg_mlp_forward_host(self._h, _u16(f), f.shape[0], _dptr(out)))
        return out

    def gradient(self, feat_bits: np.ndarray, target: np.ndarray):
        f = np.ascontiguousarray(feat_bits, dtype=np.uint16).reshape(-1, MLP_IN)
        t = np.ascontiguousarray(target, dtype=np.float32).reshape(-1, MLP_OUT)
        loss = C.c_float()
        g = np.zeros(self.param_count(), dtype=np.float32)
        check(lib().cfdg_mlp_gradient_host(self._h, _u16(f), _f32(t), f.shape[0], C.byref(loss), _f32(g)))
        return float(loss.value), g

    def train(self, ds: "Dataset", epochs: int = 1, batch: int = 4096, lr: float = 1e-3, seed: int = 7) -> float:
        loss = C.c_float()
        check(lib().cfdg_mlp_train(self._h, ds._h, epochs, batch, lr, seed, C.byref(loss)))
        return float(loss.value)


class Dataset:
    """cfdg_dataset: device buffer of (features, normalised dU) samples."""

    def __init__(self, nvars: int, capacity: int, device: int = 0):
        h = C.c_void_p()
        check(lib().cfdg_dataset_create(device, nvars, capacity, C.byref(h)))
        self._h = h
        self.nvars = nvars
        self.capacity = capacity

    def close(self):
        if getattr(self, "_h", None):
            lib().cfdg_dataset_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        n = C.c_int64()
        check(lib().cfdg_dataset_size(self._h, C.byref(n)))
        return int(n.value)

    def clear(self):
        check(lib().cfdg_dataset_clear(self._h))

    def append(self, feat_bits, target):
        f = np.ascontiguousarray(feat_bits, dtype=np.uint16).reshape(-1, MLP_IN)
        t = np.ascontiguousarray(target, dtype=np.float32).reshape(-1, MLP_OUT)
        check(lib().cfdg_dataset_append_host(self._h, _u16(f), _f32(t), f.shape[0]))

    def read(self, rows: int | None = None):
        rows = len(self) if rows is None else rows
        f = np.zeros((rows, MLP_IN), dtype=np.uint16)
        t = np.zeros((rows, MLP_OUT), dtype=np.float32)
        check(lib().cfdg_dataset_read_host(self._h, _u16(f), _f32(t), rows))
        return f, t


def _ptr_array(ptrs):
    arr = (C.c_void_p * len(ptrs))(*[C.c_void_p(int(p)) for p in ptrs])
    return arr


class Recon:
    """cfdg_recon: GradientOperator::apply_set and Muscl::compute_limiters
    on caller-owned device arrays (integer device addresses, one per
    variable, n_cells doubles each)."""

    def __init__(self, mesh: HostMesh, gradient: int = GRAD_LSQ_NODE, limiter: int = LIM_VENKATAKRISHNAN,
                 venkat_k: float = 0.5, device: int = 0):
        h = C.c_void_p()
        check(lib().cfdg_recon_create(device, C.byref(mesh.view), gradient, limiter, venkat_k, C.byref(h)))
        self._h = h
        self.mesh = mesh

    def close(self):
        if getattr(self, "_h", None):
            lib().cfdg_recon_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def gradient(self, q, gx, gy, gz, stream: int = 0):
        n = len(q)
        check(lib().cfdg_gradient(self._h, _ptr_array(q), _ptr_array(gx), _ptr_array(gy), _ptr_array(gz), n,
                                  C.c_void_p(stream or None)))

    def limiter(self, q, gx, gy, gz, phi, stream: int = 0):
        n = len(q)
        check(lib().cfdg_limiter(self._h, _ptr_array(q), _ptr_array(gx), _ptr_array(gy), _ptr_array(gz),
                                 _ptr_array(phi), n, C.c_void_p(stream or None)))


class Bsr:
    """cfdg_bsr: BsrMatrix + SgsPreconditioner + BiCGSTAB on the device."""

    def __init__(self, row_ptr, cols, bs: int, precision: int = PREC_FP64, device: int = 0):
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        self.cols = np.ascontiguousarray(cols, dtype=np.int32)
        self.n = len(self.row_ptr) - 1
        self.bs = bs
        h = C.c_void_p()
        check(lib().cfdg_bsr_create(device, self.n, bs, self.row_ptr.ctypes.data_as(_ip),
                                    self.cols.ctypes.data_as(_ip), precision, C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().cfdg_bsr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_values(self, vals):
        v = np.ascontiguousarray(vals, dtype=np.float64)
        check(lib().cfdg_bsr_set_values(self._h, _dptr(v)))

    def spmv(self, x, y=None, alpha=1.0, beta=0.0):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros_like(x) if y is None else np.array(y, dtype=np.float64, copy=True)
        check(lib().cfdg_bsr_spmv_host(self._h, _dptr(x), _dptr(y), alpha, beta))
        return y

    def sgs_setup(self, ordering=SGS_COLOR, sweeps=1):
        check(lib().cfdg_sgs_setup(self._h, ordering, sweeps))

    def sgs_apply(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        z = np.zeros_like(r)
        check(lib().cfdg_sgs_apply_host(self._h, _dptr(r), _dptr(z)))
        return z

    def bicgstab(self, b, x0=None, precond=PC_SGS, rel_tol=1e-8, abs_tol=1e-30, max_it=500):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        r = KrylovResult()
        check(lib().cfdg_bicgstab_host(self._h, precond, rel_tol, abs_tol, max_it, _dptr(x), _dptr(b), C.byref(r)))
        return x, r

    def gmres(self, b, x0=None, precond=PC_SGS, rel_tol=1e-8, abs_tol=1e-30, max_it=500, restart=30):
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64, copy=True)
        r = KrylovResult()
        check(lib().cfdg_gmres_host(self._h, precond, rel_tol, abs_tol, max_it, restart, _dptr(x), _dptr(b),
                                    C.byref(r)))
        return x, r


from . import cases  # noqa: E402,F401  (benchmark workloads)
from . import halo  # noqa: E402,F401  (partitions and halo exchange)
