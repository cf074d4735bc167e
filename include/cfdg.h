/*
 * cfdg.h — C ABI of the B200 implementation of the implicit compressible
 * finite-volume hot path (residual R(U) -> 5x5/6x6 BSR Jacobian ->
 * BiCGSTAB + SGS -> Newton update) on one GPU holding the whole mesh.
 *
 * Conventions
 *   - Every entry point returns an int status: CFDG_OK (0) or a negative
 *     CFDG_ERR_* code; nothing aborts the process.  cfdg_status_string()
 *     names a code, cfdg_last_error() gives the last message of this thread.
 *   - Pointers whose name ends in _h are HOST buffers, _d are DEVICE
 *     buffers.  Host buffers are read or written during the call only.
 *   - Handles are thread-compatible (one handle per host thread at a time).
 *   - Field layout is SoA: one array per variable.  Linear-system vectors
 *     (right-hand side b, update du) are AoS in block order c*bs+v, as in
 *     the reference implicit integrator.
 *
 * Each declaration cites the reference interface it replaces
 * (paths inside maksim-movsisyan/Distributed-cfd-solver).
 */
#ifndef CFDG_H
#define CFDG_H

#include <stdint.h>

#if defined(__GNUC__)
#define CFDG_API __attribute__((visibility("default")))
#else
#define CFDG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define CFDG_OK               0
#define CFDG_ERR_INVALID     (-1)  /* bad argument / handle / size          */
#define CFDG_ERR_CUDA        (-2)  /* CUDA runtime error (message kept)      */
#define CFDG_ERR_NOMEM       (-3)  /* device or host allocation failed       */
#define CFDG_ERR_SINGULAR    (-4)  /* singular diagonal block in SGS setup   */
#define CFDG_ERR_NONFINITE   (-5)  /* NaN/Inf detected in residual or state  */
#define CFDG_ERR_DIVERGED    (-6)  /* Krylov breakdown                       */
#define CFDG_ERR_MESH        (-7)  /* mesh fails a geometric/topology check  */
#define CFDG_ERR_UNSUPPORTED (-8)  /* option not built                       */
#define CFDG_ERR_NODEVICE    (-9)  /* no CUDA device visible                 */

/* ------------------------------------------------------------ enumerations */
/* Cell/face types: values of mesh::CellType (include/cfd/mesh/cgnstables.hpp:20-27). */
enum { CFDG_TET = 0, CFDG_PYRA = 1, CFDG_PRISM = 2, CFDG_HEXA = 3, CFDG_TRI = 4, CFDG_QUAD = 5 };

/* BC kinds: values of bc::physical::BCType (include/cfd/bc/physical/physical_bc.hpp:12-23). */
enum {
    CFDG_BC_SUPERSONIC_INLET = 0,
    CFDG_BC_SUPERSONIC_OUTLET = 1,
    CFDG_BC_SUBSONIC_INLET = 2,
    CFDG_BC_SUBSONIC_OUTLET = 3,
    CFDG_BC_SLIP_WALL = 4,
    CFDG_BC_NO_SLIP_WALL = 5,
    CFDG_BC_NO_SLIP_WALL_HEAT_FLUX = 6,
    CFDG_BC_SYMMETRY = 7,
    CFDG_BC_FARFIELD = 8
};
/* Inflow parameterisation: bc::physical::InflowMode (physical_bc.hpp:25-29). */
enum { CFDG_INFLOW_VELOCITY = 0, CFDG_INFLOW_MACH_ANGLES = 1, CFDG_INFLOW_MACH_DIRECTION = 2 };

/* Gradient operators: numerics::gradient::GradientType
 * (include/cfd/numerics/gradient/gradient_manager.hpp:14-19); the two
 * least-squares stencils are built (Green-Gauss is not on this path). */
enum { CFDG_GRAD_LSQ_FACE = 2, CFDG_GRAD_LSQ_NODE = 3 };
/* Reconstruction: ReconType (include/cfd/solver/compressible/config.hpp). */
enum { CFDG_RECON_FIRST_ORDER = 0, CFDG_RECON_MUSCL = 1 };
/* Multidimensional limiters: LimiterType (config.hpp) / slope_limiters.hpp. */
enum { CFDG_LIM_VENKATAKRISHNAN = 1, CFDG_LIM_BARTH_JESPERSEN = 2, CFDG_LIM_VAN_ALBADA = 3 };
/* SGS sweep ordering.  LEVEL reproduces the sequential sweep of
 * linalg/bsr_helpers.hpp:389-435 exactly (level-scheduled); COLOR sweeps a
 * multicolour ordering (a different, equally valid SGS preconditioner). */
enum { CFDG_SGS_LEVEL = 0, CFDG_SGS_COLOR = 1 };
/* Matrix precision: FP64 everywhere, or FP32 Jacobian/LU/SpMV/SGS with FP64
 * vectors, residual, update and inner products. */
enum { CFDG_PREC_FP64 = 0, CFDG_PREC_MIXED = 1 };
/* Preconditioner: linalg::PreconditionerType (linalg/config.hpp:12). */
enum { CFDG_PC_NONE = 0, CFDG_PC_SGS = 1 };
/* Krylov status: linalg::SolverStatus (linalg/types.hpp). */
enum { CFDG_KRYLOV_CONVERGED = 0, CFDG_KRYLOV_DIVERGED = 1, CFDG_KRYLOV_MAX_ITERATIONS = 2 };

/* Fields readable with cfdg_solver_get_field (sizes in doubles). */
enum {
    CFDG_FIELD_U = 0,        /* conserved state, nvars x n_cells                  */
    CFDG_FIELD_Q = 1,        /* primitives (p,u,v,w,T), 5 x n_total (ghosts incl.)*/
    CFDG_FIELD_GRAD = 2,     /* gradients, (5|6) vars x 3 planes x n_total        */
    CFDG_FIELD_PHI = 3,      /* limiter, 5 x n_cells                              */
    CFDG_FIELD_RES = 4,      /* residual, nvars x n_cells                         */
    CFDG_FIELD_LAM = 5,      /* spectral radius, n_cells                          */
    CFDG_FIELD_DT = 6,       /* local time step, n_cells                          */
    CFDG_FIELD_ALPHA = 7,    /* diagonal shift V/dt, n_cells                      */
    CFDG_FIELD_JAC = 8,      /* BSR values, nnzb x bs x bs (row-major blocks)     */
    CFDG_FIELD_DU = 9,       /* last Newton update, AoS n_cells x nvars           */
    CFDG_FIELD_MUT = 10,     /* eddy viscosity, n_total (SA only)                 */
    CFDG_FIELD_WALLDIST = 11,/* wall distance, n_cells (SA only)                  */
    CFDG_FIELD_RHS = 12,     /* linear right-hand side -R, AoS n_cells x nvars    */
    CFDG_FIELD_NU = 13,      /* specific nu_tilde, n_cells (SA only)              */
    CFDG_FIELD_NU_GRAD = 14  /* nu_tilde gradient, 3 planes x n_total (SA only)  */
};

/* Pipeline stages for cfdg_solver_stage (each is one step of
 * Solver::evaluate_residual, include/cfd/solver/compressible/solver.hpp:169-247). */
enum {
    CFDG_STAGE_PRIMITIVES = 0,  /* step 1 + BC ghost values (steps 1,3)         */
    CFDG_STAGE_GRADIENT = 1,    /* step 5: gradient operator on owned cells       */
    CFDG_STAGE_LIMITER = 2,     /* step 5: ghost gradients + MUSCL limiter        */
    CFDG_STAGE_FLUXES = 3       /* step 6 (+ SA steps 7,8): face sweep -> R, lam  */
};

/* Kernel families timed by the optional profiler (CUDA events on the
 * solver stream around every launch of the family). */
enum {
    CFDG_KCAT_PRIMITIVES = 0, CFDG_KCAT_GRADIENT = 1, CFDG_KCAT_LIMITER = 2, CFDG_KCAT_FACE_FLUX = 3,
    CFDG_KCAT_CELL_GATHER = 4, CFDG_KCAT_JACOBIAN = 5, CFDG_KCAT_LU = 6, CFDG_KCAT_SPMV = 7, CFDG_KCAT_SGS = 8,
    CFDG_KCAT_KRYLOV = 9, CFDG_KCAT_UPDATE = 10, CFDG_KCAT_TURBULENCE = 11,
    CFDG_KCAT_GUESS = 12, CFDG_KCAT_JFNK = 13, CFDG_KCAT_COUNT = 14
};

/* ------------------------------------------------------------- structures */
/* Host view of one single-partition mesh with geometry, the subset of
 * mesh::MeshPart (include/cfd/mesh/localmesh.hpp:17-102) the solver reads.
 * Faces follow the reference 3-zone order: interior faces [0,n_inner_faces)
 * sorted by (owner, neigh), then boundary faces sorted by (patch, owner);
 * the BC ghost of boundary face f is slot n_cells + (f - n_inner_faces). */
typedef struct cfdg_mesh_host {
    int32_t n_cells, n_faces, n_inner_faces, n_nodes, n_patches;
    const uint8_t* cell_type;           /* n_cells                           */
    const int32_t* cell_nodes_offsets;  /* n_cells+1                         */
    const int32_t* cell_nodes;          /* CGNS node order                   */
    const double *node_x, *node_y, *node_z;
    const double *cell_centroid_x, *cell_centroid_y, *cell_centroid_z, *cell_volume;
    const int32_t *face_owner, *face_neigh, *face_patch;  /* neigh=-1, patch=-1 */
    const int32_t *face_nodes_offsets, *face_nodes;
    const double *face_centroid_x, *face_centroid_y, *face_centroid_z;
    const double *face_normal_x, *face_normal_y, *face_normal_z, *face_area;
} cfdg_mesh_host;

/* One boundary patch: bc::BCDescriptor (include/cfd/bc/config.hpp). */
typedef struct cfdg_bc_desc {
    int32_t patch_id, type, inflow_mode, pad_;
    double p, t, tmp_grad;
    double velocity[3];
    double mach, alpha_deg, beta_deg;
    double direction[3];
} cfdg_bc_desc;

/* Viscous part of the Picard Jacobian.  REFERENCE: the reference's
 * thin-layer block mu/d * I on the velocity, boundary faces against a frozen
 * ghost (viscous.hpp:280-360, jacobian_kernel.hpp:232-269).  THIN_LAYER:
 * mu/d * (I + n n^T / 3) (the normal-stress term) and, on no-slip wall
 * faces, the ghost's mirrored velocity (isothermal: temperature) doubling
 * the owner derivative; the residual is the same. */
enum { CFDG_JAC_REFERENCE = 0, CFDG_JAC_THIN_LAYER = 1 };

/* BiCGSTAB iteration driver (cfdg_config.krylov_loop). */
enum { CFDG_KRYLOV_DEVICE_LOOP = 0, CFDG_KRYLOV_HOST_LOOP = 1 };

/* Time mode (cfdg_config.time_mode). */
enum { CFDG_TIME_STEADY = 0, CFDG_TIME_UNSTEADY = 1 };

/* Linear solves before the limiter freeze (cfdg_config.pre_freeze).
 * CONFIGURED: the configured matrix precision and initial guess throughout.
 * FP64: until the limiter is frozen the linear solves use the FP64 matrix
 * and start from zero (no learned guess), so the iterates up to the freeze
 * are bitwise those of the plain FP64 path, the frozen limiter is the same,
 * and a mixed-precision / learned-guess run converges to the FP64 run's
 * discrete solution (the switching limiter makes the state at the freeze,
 * and with it the frozen problem, depend on every rounding before it). */
enum { CFDG_PREFREEZE_CONFIGURED = 0, CFDG_PREFREEZE_FP64 = 1 };

/* Newton operator (cfdg_config.newton_operator).  PICARD: the Krylov
 * products use the assembled first-order matrix, as the reference's
 * BackwardEuler does (time/implicit_euler.hpp:34-76).  JACOBIAN_FREE (not in
 * the reference): once the limiter is frozen (from the first iteration
 * without MUSCL) the products are the directional derivative of the full
 * second-order residual, v -> (V/dt) v + (R(U + eps v) - R(U)) / eps, with
 * one eps per product that moves no conserved variable by more than
 * jf_eps of its RMS; SGS on the assembled matrix stays the preconditioner.
 * A Jacobian-free solve that does not bring its residual below jf_accept
 * ||b|| is replaced by the Picard solve of the same step, and a
 * Jacobian-free step is relaxed
 * so that rho and rho E (and rho nu~, against |rho nu~| + 1e-3 of its RMS)
 * change by at most jf_max_change in any cell.  The residual, and with it
 * the converged state, is the same; only the path to it changes. */
enum { CFDG_NEWTON_PICARD = 0, CFDG_NEWTON_JACOBIAN_FREE = 1 };

/* Krylov method of the Jacobian-free solves (cfdg_config.jf_krylov):
 * BiCGSTAB as for the Picard matrix, or restarted GMRES(jf_restart) with
 * right preconditioning, whose residual never grows. */
enum { CFDG_JF_BICGSTAB = 0, CFDG_JF_GMRES = 1 };

/* Solver configuration: SolverConfig + linalg::SolverParams
 * (include/cfd/solver/compressible/config.hpp:94-136, linalg/config.hpp:14-26)
 * plus the CFL ramp, precision, SGS ordering, SA and learned-guess options. */
typedef struct cfdg_config {
    int32_t viscous;          /* 0 Euler (InviscidFlow), 1 Navier-Stokes      */
    int32_t turbulence;       /* 0 none, 1 Spalart-Allmaras (6 variables)     */
    int32_t gradient;         /* CFDG_GRAD_*                                  */
    int32_t reconstruction;   /* CFDG_RECON_*                                 */
    int32_t limiter;          /* CFDG_LIM_*                                   */
    int32_t precision;        /* CFDG_PREC_*                                  */
    int32_t precond;          /* CFDG_PC_*                                    */
    int32_t sgs_ordering;     /* CFDG_SGS_*                                   */
    int32_t sgs_sweeps;       /* >= 1                                         */
    int32_t lin_max_iterations;
    int32_t cfl_ramp_iterations; /* iterations over which CFL goes cfl->cfl_max */
    int32_t residual_interval;
    /* 0: the reference monitor, max over variables of L2_v / L2_v(first
     *    diagnosed iteration) (solver.hpp:631-636,758-765);
     * 1: max over (mass, |momentum|, energy[, nu_tilde]) of L2 / running
     *    maximum of L2 (robust when a component starts at round-off, e.g.
     *    spanwise momentum of a quasi-2-D case or a uniform initial state). */
    int32_t convergence_monitor;
    int32_t jacobian;         /* CFDG_JAC_*                                   */
    /* run_steady freezes the MUSCL limiter values from this iteration on
     * (0 = never); cfdg_solver_freeze_limiter does it from the host loop */
    int32_t limiter_freeze;
    /* CFDG_KRYLOV_DEVICE_LOOP: the BiCGSTAB iterations run as one CUDA graph
     * whose conditional while-node repeats the iteration until the device-side
     * state stops it (no host round trip per iteration; profiling switches to
     * the host loop); CFDG_KRYLOV_HOST_LOOP: one launch sequence per
     * iteration with the host reading the state after each. */
    int32_t krylov_loop;
    int32_t pre_freeze;       /* CFDG_PREFREEZE_*                             */
    int32_t reserved_;        /* zero                                         */
    double gamma, gas_constant, prandtl, prandtl_turb;
    double init_rho, init_p, init_velocity[3];
    double venkat_k;
    double cfl, cfl_max;
    double residual_tolerance;
    double lin_rel_tol, lin_abs_tol;
    double nu_inf_ratio;      /* SA freestream nu_tilde / nu                   */
    int64_t max_iterations;   /* steady: iterations; unsteady: sub-iterations per time step */
    /* Dual time stepping (TimeMode::Unsteady, include/cfd/solver/time_mode.hpp;
     * SolverConfig [time] dt, max_time_steps, bdf_order): time_mode
     * CFDG_TIME_STEADY or CFDG_TIME_UNSTEADY, BDF order 1 or 2 (the first
     * physical step is BDF1), physical step dt_physical [s]. */
    double dt_physical;
    int64_t max_time_steps;
    int32_t time_mode;
    int32_t bdf_order;
    int32_t newton_operator;  /* CFDG_NEWTON_*                                */
    int32_t jf_max_iterations; /* Krylov cap of a Jacobian-free solve          */
    double jf_rel_tol;        /* relative tolerance of a Jacobian-free solve   */
    double jf_eps;            /* product step: fraction of each variable's RMS */
    double jf_max_change;     /* relaxation of Jacobian-free steps (0: off)    */
    /* Switched evolution relaxation after the CFL ramp (run_steady):
     * CFL = cfl_max * max(1, rel at the ramp's end / rel of the last
     * iteration), at most cfl_ser_max; off when cfl_ser_max <= cfl_max. */
    double cfl_ser_max;
    int32_t jf_krylov;        /* CFDG_JF_*                                    */
    int32_t jf_restart;       /* GMRES restart length, 1..200                 */
    /* a Jacobian-free solve is kept when its residual is at most jf_accept
     * x ||b||; otherwise the Picard solve of the step replaces it */
    double jf_accept;
} cfdg_config;

typedef struct cfdg_krylov_result {
    int32_t status;            /* CFDG_KRYLOV_*                              */
    int32_t iterations;
    double initial_residual, final_residual;
} cfdg_krylov_result;

typedef struct cfdg_step_result {
    double l2[6];              /* L2 residual norms of the evaluated R(U)    */
    double cfl;
    int32_t nvars;
    int32_t krylov_status, krylov_iterations;
    int32_t guess_used;        /* 0 zero guess, 1 learned guess, 2 learned guess rejected */
    double krylov_initial, krylov_final;
    double krylov_rhs;         /* ||b||: krylov_initial / krylov_rhs < 1 when the guess helped */
    int32_t jacobian_free;     /* 1: the update came from a Jacobian-free solve */
    int32_t picard_fallback;   /* 1: a Jacobian-free solve failed and the Picard solve replaced it */
    double step_scale;         /* relaxation factor applied to the update (1: none) */
} cfdg_step_result;

typedef struct cfdg_run_result {
    int64_t iterations;
    int32_t converged, blowup;
    double rel, seconds;
    int64_t krylov_iterations_total;
    double l2_first[6], l2_last[6];
    int64_t jacobian_free_steps;      /* updates from Jacobian-free solves    */
    int64_t picard_fallbacks;         /* Jacobian-free solves replaced by Picard */
    double cfl_last;                  /* CFL of the last iteration            */
} cfdg_run_result;

typedef struct cfdg_unsteady_result {
    int64_t time_steps;               /* physical steps taken                    */
    int64_t subiterations_total;      /* Newton sub-iterations over all steps    */
    int64_t krylov_iterations_total;
    int32_t steps_converged;          /* steps whose sub-iterations met the tolerance */
    int32_t blowup;
    double t_physical, seconds;
    double l2_last[6];                /* norms of the last sub-iteration's residual */
} cfdg_unsteady_result;

typedef struct cfdg_solver cfdg_solver;   /* Solver<...> + BackwardEuler     */
typedef struct cfdg_bsr cfdg_bsr;         /* BsrMatrix + SGS + BiCGSTAB      */
typedef struct cfdg_host_mesh cfdg_host_mesh;
typedef struct cfdg_mlp cfdg_mlp;         /* learned initial-guess network    */
typedef struct cfdg_dataset cfdg_dataset; /* (features, dU) training samples  */

/* ------------------------------------------------------------ library */
CFDG_API int cfdg_version(void);
CFDG_API const char* cfdg_status_string(int status);
CFDG_API const char* cfdg_last_error(void);
CFDG_API int cfdg_device_count(int* count_h);
CFDG_API void cfdg_config_default(cfdg_config* cfg_h);

/* ------------------------------------------------------- synthetic meshes */
/* Generates the benchmark meshes in memory, replacing the CGNS/HDF5 import
 * (apps/solver.cpp:89, io::solver_mesh::import_mesh_hdf5) that cannot be
 * built here.  kind: 0 = compression-ramp hex block, 1 = flat-plate hex
 * block, 2 = tetrahedral bump.  Cells are permuted by a seeded shuffle and
 * renumbered by reverse Cuthill-McKee (the ordering of
 * mesh::reorder_local_mesh(RCM), src/mesh/reorder.cpp:135-190,579-602);
 * geometry follows mesh::compute_mesh_geometry (src/mesh/geometry.cpp:301-540). */
typedef struct cfdg_mesh_spec {
    int32_t kind, nx, ny, nz;
    double lx, ly, lz;           /* domain extents [m]                          */
    double first_spacing;        /* wall-normal first cell height (plate) [m]  */
    double stretch;              /* wall-normal growth ratio (plate)           */
    double cap_spacing;          /* stop growth at this spacing (0 = never)    */
    double jitter;               /* interior node jitter, fraction of spacing  */
    double ramp_angle_deg, ramp_x;   /* ramp geometry                          */
    double plate_x0;             /* plate leading edge x (symmetry before it)  */
    double bump_height, bump_x0, bump_x1;
    uint64_t seed;
    int32_t permute, reorder_rcm;
} cfdg_mesh_spec;
CFDG_API int cfdg_mesh_generate(const cfdg_mesh_spec* spec_h, cfdg_host_mesh** out);
CFDG_API int cfdg_host_mesh_view(const cfdg_host_mesh* mesh, cfdg_mesh_host* view_h);
CFDG_API int cfdg_host_mesh_free(cfdg_host_mesh* mesh);
/* Recomputes cell/face geometry of a view in place of the arrays it points
 * to (compute_mesh_geometry, src/mesh/geometry.cpp:301-540). */
CFDG_API int cfdg_mesh_compute_geometry(cfdg_host_mesh* mesh);

/* ----------------------------------------------------------- solver */
/* Solver ctor (solver.hpp:74-150): uploads the mesh, builds connectivity,
 * LSQ coefficients, BSR structure and SGS orderings, allocates device state. */
CFDG_API int cfdg_solver_create(int device, const cfdg_mesh_host* mesh_h, const cfdg_config* cfg_h,
                       const cfdg_bc_desc* bcs_h, int32_t n_bcs, cfdg_solver** out);
CFDG_API int cfdg_solver_destroy(cfdg_solver* s);
/* Solver::init_fields (solver.hpp:507-544): uniform [initial] state. */
CFDG_API int cfdg_solver_init_fields(cfdg_solver* s);
/* Sets the conserved state from host SoA arrays (nvars x ld doubles, cells 0..n_cells). */
CFDG_API int cfdg_solver_set_state(cfdg_solver* s, const double* u_h, int64_t ld);
CFDG_API int cfdg_solver_get_field(cfdg_solver* s, int32_t field, double* out_h, int64_t count);
CFDG_API int cfdg_solver_sizes(const cfdg_solver* s, int64_t* sizes_h /* n_cells,n_faces,n_inner,n_total,nnzb,bs,nvars */);
/* Solver::evaluate_residual (solver.hpp:169-247). */
CFDG_API int cfdg_evaluate_residual(cfdg_solver* s);
CFDG_API int cfdg_solver_stage(cfdg_solver* s, int32_t stage);
/* Solver::compute_dt (solver.hpp:256-287) with the given CFL. */
CFDG_API int cfdg_compute_dt(cfdg_solver* s, double cfl);
/* Solver::assemble_jacobian -> JacobianKernel::apply (jacobian_kernel.hpp:74-103). */
CFDG_API int cfdg_assemble_jacobian(cfdg_solver* s);
/* set_rhs_and_zero_du + BSRLinearSystem::solve (implicit_euler.hpp:81-92,
 * bsr_linear_system.hpp:93-97). */
CFDG_API int cfdg_linear_solve(cfdg_solver* s, cfdg_krylov_result* out_h);
/* BackwardEuler::advance (implicit_euler.hpp:34-76) at the given CFL. */
CFDG_API int cfdg_newton_step(cfdg_solver* s, double cfl, cfdg_step_result* out_h);
/* Freezes (1) or releases (0) the MUSCL limiter values: while frozen the
 * residual reuses the last computed phi (a smooth residual for the final
 * orders of convergence; not in the reference, which recomputes it). */
CFDG_API int cfdg_solver_freeze_limiter(cfdg_solver* s, int32_t frozen);
/* Loads limiter values (5 x n_cells, SoA as CFDG_FIELD_PHI) and freezes
 * them: two runs given the same values converge to the same discrete
 * solution. */
CFDG_API int cfdg_solver_set_limiter(cfdg_solver* s, const double* phi_h, int64_t count);
/* Solver::residual_norms (solver.hpp:740-756), nvars doubles. */
CFDG_API int cfdg_residual_norms(cfdg_solver* s, double* l2_h);
/* Allocation-free variant of cfdg_residual_norms, with no counterpart in the
 * reference: per-variable L2 norms sqrt(sum_c r_v[c]^2 / n_cells) of an SoA
 * device array (nvars x n_cells doubles) the caller owns, for callers that
 * cannot allocate device memory (a host code whose pool owns the whole device
 * budget, or a hook between solver kernels where cudaMalloc would
 * synchronise).  Scratch is a static 768 KiB device array: nvars <= 6 and
 * n_cells <= 4,194,304, larger sizes return CFDG_ERR_INVALID.  stream may be
 * NULL (legacy default stream); the call synchronises it.  Calls share the
 * scratch, so calls that overlap on the GPU race; the first call on a device
 * looks up the scratch address there and should come before any stream
 * capture.  The address is kept for the life of the process: after a
 * cudaDeviceReset (or anything else that re-creates the device's primary
 * context) the entry point must not be called again in that process. */
CFDG_API int cfdg_residual_norms_noalloc(const double* res_d, int32_t n_cells, int32_t nvars, void* stream,
                                         double* l2_h);
/* Solver::run_steady (solver.hpp:597-660) with the CFL ramp. */
CFDG_API int cfdg_run_steady(cfdg_solver* s, cfdg_run_result* out_h);
/* Solver::run_dual_time (solver.hpp:662-736), cfg.time_mode ==
 * CFDG_TIME_UNSTEADY: max_time_steps physical steps of dt_physical, each
 * up to max_iterations Newton sub-iterations of the residual with the BDF
 * pseudo-source (add_unsteady_source_term, solver.hpp:546-580) and the
 * V c0 / dt diagonal (compute_dt, solver.hpp:267-277), stopped when the
 * monitor (checked on sub-iteration 1, every 5th and the last) drops below
 * residual_tolerance; then U^{n-1} <- U^n, U^n <- U
 * (shift_physical_time_levels, solver.hpp:582-596). */
CFDG_API int cfdg_run_unsteady(cfdg_solver* s, cfdg_unsteady_result* out_h);
/* Solver::write_fields (solver.hpp:856-898) via io::vtk::write_solution_vtu
 * (src/io/vtk/vtu.cpp:321-470) at one rank: writes <outdir>/<stem>_00000.vtu
 * (ASCII VTK unstructured grid: the mesh's points and cells, CellData rank,
 * rho, u, v, w, pressure, mach, and with Spalart-Allmaras nu_tilde and mu_t)
 * and <outdir>/<stem>.pvtu.  The fields are formed on the device from the
 * current state; mesh_h must be the mesh the solver was created with. */
CFDG_API int cfdg_solver_write_vtu(cfdg_solver* s, const cfdg_mesh_host* mesh_h, const char* outdir,
                                   const char* stem);
/* U^n = U^{n-1} = U: the physical time levels of the current state
 * (init_fields does this; call it after cfdg_solver_set_state). */
CFDG_API int cfdg_solver_reset_time_levels(cfdg_solver* s);
/* Stream all solver kernels are queued on (cudaStream_t as void*). */
CFDG_API void* cfdg_solver_stream(cfdg_solver* s);
/* Total solver kernel launches since creation (for launch accounting). */
CFDG_API int64_t cfdg_solver_launch_count(const cfdg_solver* s);
/* Enables (1) or disables (0) per-launch CUDA-event timing; resets counters. */
CFDG_API int cfdg_solver_profile(cfdg_solver* s, int32_t enable);
/* Accumulated device milliseconds, launch counts and algorithmic
 * (unique-touch) bytes per CFDG_KCAT_* family; bytes_h may be NULL. */
CFDG_API int cfdg_solver_profile_read(cfdg_solver* s, double* ms_h, int64_t* launches_h, double* bytes_h);
/* Number of SGS colours / forward levels of the active ordering. */
CFDG_API int cfdg_solver_sgs_info(const cfdg_solver* s, int32_t* n_groups_fwd_h, int32_t* n_groups_bwd_h);

/* ------------------------------------------ gradient and limiter operators
 * The reconstruction steps of the residual on fields the caller owns, for
 * callers that keep their own state (the GradientOperator and
 * ReconstructionPolicy seams of the reference).  Fields are device arrays
 * of n_cells doubles, one per variable; q_d, gx_d, gy_d, gz_d and phi_d are
 * HOST arrays of nvars such device pointers.  At one partition the cells
 * are the owned cells and no BC ghost enters either stencil (as in the
 * reference).  Launches are queued on `stream` (NULL: legacy default
 * stream) and the calls return without synchronising. */
typedef struct cfdg_recon cfdg_recon;
/* GradientOperator::setup (include/cfd/numerics/gradient/gradient_operator.hpp:16-44,
 * LSQ set-up src/numerics/gradient/gradient_operator.cpp:414-499,622-707)
 * plus the limiter's face connectivity: gradient CFDG_GRAD_LSQ_FACE or
 * CFDG_GRAD_LSQ_NODE, limiter CFDG_LIM_*, venkat_k the Venkatakrishnan K. */
CFDG_API int cfdg_recon_create(int device, const cfdg_mesh_host* mesh_h, int32_t gradient, int32_t limiter,
                               double venkat_k, cfdg_recon** out);
CFDG_API int cfdg_recon_destroy(cfdg_recon* r);
/* GradientOperator::apply_set (gradient_operator.hpp:38-43): the gradient of
 * each q_d[v] on the cells into gx_d[v], gy_d[v], gz_d[v]. */
CFDG_API int cfdg_gradient(cfdg_recon* r, const double* const* q_d, double* const* gx_d, double* const* gy_d,
                           double* const* gz_d, int32_t nvars, void* stream);
/* Muscl<Limiter>::compute_limiters (include/cfd/numerics/reconstruction/muscl.hpp:25-105):
 * phi_d[v] from q_d[v] and its gradient (face-neighbour extrema, minimum of
 * the limiter function over the cell's faces). */
CFDG_API int cfdg_limiter(cfdg_recon* r, const double* const* q_d, const double* const* gx_d,
                          const double* const* gy_d, const double* const* gz_d, double* const* phi_d, int32_t nvars,
                          void* stream);

/* ------------------------------------------------ block-sparse linear algebra */
/* BsrMatrix + assemble (src/linalg/bsr_matrix.cpp:22-40): structure from
 * host CSR (sorted columns, diagonal present), values set later. */
CFDG_API int cfdg_bsr_create(int device, int32_t n_rows, int32_t bs, const int32_t* row_ptr_h,
                    const int32_t* cols_h, int32_t precision, cfdg_bsr** out);
CFDG_API int cfdg_bsr_destroy(cfdg_bsr* a);
CFDG_API int cfdg_bsr_set_values(cfdg_bsr* a, const double* values_h);
/* LinearOperator::apply, y = alpha*A*x + beta*y (bsr_matrix.cpp:10-20). */
CFDG_API int cfdg_bsr_spmv(cfdg_bsr* a, const double* x_d, double* y_d, double alpha, double beta);
CFDG_API int cfdg_bsr_spmv_host(cfdg_bsr* a, const double* x_h, double* y_h, double alpha, double beta);
/* Preconditioner::setup for SGS: block LU of the diagonal
 * (preconditioners.cpp:62-93). */
CFDG_API int cfdg_sgs_setup(cfdg_bsr* a, int32_t ordering, int32_t sweeps);
/* Preconditioner::apply for SGS: z = M^-1 r (preconditioners.cpp:171-194). */
CFDG_API int cfdg_sgs_apply(cfdg_bsr* a, const double* r_d, double* z_d);
CFDG_API int cfdg_sgs_apply_host(cfdg_bsr* a, const double* r_h, double* z_h);
/* IterativeSolver::solve for BiCGSTAB (src/linalg/bicgstab.cpp:42-201);
 * x holds the initial guess on entry.  precond: CFDG_PC_*. */
CFDG_API int cfdg_bicgstab(cfdg_bsr* a, int32_t precond, double rel_tol, double abs_tol, int32_t max_it,
                  double* x_d, const double* b_d, cfdg_krylov_result* out_h);
CFDG_API int cfdg_bicgstab_host(cfdg_bsr* a, int32_t precond, double rel_tol, double abs_tol, int32_t max_it,
                       double* x_h, const double* b_h, cfdg_krylov_result* out_h);
/* Restarted GMRES(restart) with right preconditioning (not in the
 * reference; the Krylov method of the Jacobian-free solves, CFDG_JF_GMRES);
 * same arguments and conventions as cfdg_bicgstab, restart in [1, 200]. */
CFDG_API int cfdg_gmres(cfdg_bsr* a, int32_t precond, double rel_tol, double abs_tol, int32_t max_it, int32_t restart,
               double* x_d, const double* b_d, cfdg_krylov_result* out_h);
CFDG_API int cfdg_gmres_host(cfdg_bsr* a, int32_t precond, double rel_tol, double abs_tol, int32_t max_it,
                    int32_t restart, double* x_h, const double* b_h, cfdg_krylov_result* out_h);

/* ------------------------------------------------ learned initial guess
 * Not in the reference (its BiCGSTAB starts from the zero vector,
 * implicit_euler.hpp:81-92; x0 != 0 is supported by bicgstab.cpp:57-60).
 * A per-cell MLP (48 features -> 64 -> 64 -> nvars, ReLU, bf16 weights,
 * fp32 accumulation on the tcgen05 tensor cores) predicts the Newton update
 * dU0 from the cell's explicit pseudo-time update, state and previous update
 * and their face-neighbour mean / max; BiCGSTAB then starts from dU0 unless
 * ||b - A dU0|| >= ||b||, in which case it starts from zero.  Parameters:
 * fp32, W1[64x48] b1[64] W2[64x64] b2[64] W3[16x64] b3[16] (row-major,
 * out x in), cfdg_mlp_param_count() values. */
/* D[128 x n] = A[128 x k] B[n x k]^T on one CTA of tensor cores (bf16 bits,
 * row-major); n in {16,32,48,64}, k a multiple of 16 <= 128. */
CFDG_API int cfdg_tc_selftest(int device, int32_t n, int32_t k, const uint16_t* a_h, const uint16_t* b_h,
                              float* d_h);
CFDG_API int cfdg_mlp_create(int device, int32_t nvars, uint64_t seed, cfdg_mlp** out);
CFDG_API int cfdg_mlp_destroy(cfdg_mlp* m);
CFDG_API int32_t cfdg_mlp_param_count(void);
CFDG_API int cfdg_mlp_get_params(cfdg_mlp* m, float* out_h, int64_t count);
CFDG_API int cfdg_mlp_set_params(cfdg_mlp* m, const float* params_h, int64_t count);
/* out[r*nvars+v] = scale[v] * y_v(row r); features bf16 bits [rows x 48] (device) */
CFDG_API int cfdg_mlp_forward(cfdg_mlp* m, const uint16_t* feat_d, int64_t rows, const double* scale_d,
                              double* out_d);
CFDG_API int cfdg_mlp_forward_host(cfdg_mlp* m, const uint16_t* feat_h, int64_t rows, double* out_h);
/* mean squared error over rows x nvars of targets t [rows x 16] and its
 * gradient (cfdg_mlp_param_count() floats); no update */
CFDG_API int cfdg_mlp_gradient_host(cfdg_mlp* m, const uint16_t* x_h, const float* t_h, int64_t rows,
                                    float* loss_h, float* grad_h);
/* Adam over the dataset (shuffled contiguous batches); mean loss of the last epoch */
CFDG_API int cfdg_mlp_train(cfdg_mlp* m, cfdg_dataset* ds, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                            float* loss_h);
CFDG_API int cfdg_dataset_create(int device, int32_t nvars, int64_t capacity, cfdg_dataset** out);
CFDG_API int cfdg_dataset_destroy(cfdg_dataset* d);
CFDG_API int cfdg_dataset_size(const cfdg_dataset* d, int64_t* size_h);
CFDG_API int cfdg_dataset_clear(cfdg_dataset* d);
CFDG_API int cfdg_dataset_append_host(cfdg_dataset* d, const uint16_t* x_h, const float* t_h, int64_t rows);
CFDG_API int cfdg_dataset_read_host(const cfdg_dataset* d, uint16_t* x_h, float* t_h, int64_t rows);
/* The solver starts each linear solve from the network's guess (NULL:
 * zero guess); a dataset receives the features and normalised solved
 * update of every stride-th cell of every Newton step until it is full. */
CFDG_API int cfdg_solver_attach_guess(cfdg_solver* s, cfdg_mlp* m);
CFDG_API int cfdg_solver_attach_dataset(cfdg_solver* s, cfdg_dataset* d, int32_t stride);

/* ---------------------------------------------------- partitions and halos
 * The halo fields of mesh::MeshPart (include/cfd/mesh/localmesh.hpp:30-32,
 * 79-83) for one rank of a partitioned mesh, and the device side of
 * HaloExchanger (src/fields/halo.cpp:212-330): pack the listed owned
 * cells of SoA fields into one AoS message (nvars values a cell, one group
 * a neighbour, in plan order) and scatter a received message into the
 * ghost cells.  The transport of the messages is the caller's (NCCL
 * send/recv, e.g. through torch.distributed); the solver itself runs one
 * partition (n_own == n_cells).
 * part_h[c]: the rank owning global cell c, or NULL for nparts contiguous
 * ranges of the cell order.  Local cells: the owned cells in ascending
 * global order, then the ghosts grouped by owning rank (ascending) and
 * ascending in global id; a sender's group for rank r lists the same cells
 * in the same order as r's group for the sender.  Host only until the
 * first pack/unpack, which uploads the index lists to `device`. */
typedef struct cfdg_halo cfdg_halo;
enum {
    CFDG_HALO_LOCAL_TO_GLOBAL = 0,   /* n_local                                */
    CFDG_HALO_NB_RANKS = 1,          /* n_neighbours                           */
    CFDG_HALO_SEND_OFFSETS = 2,      /* n_neighbours + 1                       */
    CFDG_HALO_SEND_OWNED_LOCAL = 3,  /* n_send: local indices in [0, n_own)     */
    CFDG_HALO_RECV_OFFSETS = 4,      /* n_neighbours + 1                       */
    CFDG_HALO_RECV_GHOST_LOCAL = 5   /* n_recv: local indices in [n_own, n_local) */
};
CFDG_API int cfdg_halo_create(const cfdg_mesh_host* mesh_h, int32_t nparts, const int32_t* part_h, int32_t rank,
                              cfdg_halo** out);
CFDG_API int cfdg_halo_destroy(cfdg_halo* h);
/* sizes_h[5] = {n_own, n_local, n_neighbours, n_send, n_recv} */
CFDG_API int cfdg_halo_sizes(const cfdg_halo* h, int64_t* sizes_h);
CFDG_API int cfdg_halo_get(const cfdg_halo* h, int32_t what, int32_t* out_h, int64_t count);
/* send_d[i*nvars + v] = fields_d[v][send_owned_local[i]], i < n_send;
 * fields_d is a host array of nvars (<= 32) device pointers */
CFDG_API int cfdg_halo_pack(cfdg_halo* h, int device, const double* const* fields_d, int32_t nvars, double* send_d,
                            void* stream);
/* fields_d[v][recv_ghost_local[i]] = recv_d[i*nvars + v], i < n_recv */
CFDG_API int cfdg_halo_unpack(cfdg_halo* h, int device, const double* recv_d, int32_t nvars,
                              double* const* fields_d, void* stream);
/* The same for a block vector x_d[row*bs + v] (n_local rows, local order;
 * the Krylov vectors' layout, vector_layout.hpp:170-250), bs in [1, 32]:
 * send_d[i*bs + v] = x_d[send_owned_local[i]*bs + v] and
 * x_d[recv_ghost_local[i]*bs + v] = recv_d[i*bs + v]. */
CFDG_API int cfdg_halo_pack_blocks(cfdg_halo* h, int device, const double* x_d, int32_t bs, double* send_d,
                                   void* stream);
CFDG_API int cfdg_halo_unpack_blocks(cfdg_halo* h, int device, const double* recv_d, int32_t bs, double* x_d,
                                     void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CFDG_H */
