// Device-side data views and launch helpers shared by all kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cfdg {

constexpr int kMaxVars = 6;

// Per-patch boundary data resolved on the host from bc::BCDescriptor the way
// BoundaryManager::register_all does (include/cfd/solver/compressible/bc_manager.hpp:223-329).
struct BcPatch {
    int32_t kind;   // CFDG_BC_* (or -1: patch absent from the configuration)
    int32_t sa_kind;  // nu_tilde treatment: 0 wall, 1 inflow, 2 outflow, 3 symmetry
    double qfix[5];   // fixed primitive state (p,u,v,w,T) where the BC has one
    double p_out;     // subsonic outlet back pressure
    double tmp_grad;  // heat-flux wall normal temperature gradient
    double far_p, far_T, far_u, far_v, far_w;  // farfield freestream
};

// Read-only mesh arrays on the device (single partition, n_own == n_cells).
struct DevMesh {
    int32_t n, nf, ni, nb, nt;           // cells, faces, inner faces, boundary faces, n + nb
    const int32_t* owner;                // nf
    const int32_t* neigh;                // nf
    const int32_t* bpatch;               // nb: patch of face ni + b
    const double *fnx, *fny, *fnz, *farea;      // nf
    const double *fcx, *fcy, *fcz;              // nf
    const double *fdx, *fdy, *fdz, *finv_d;     // nf: face-cell distance vectors, 1/|d|
    const double *ccx, *ccy, *ccz, *vol;        // n
    const int32_t *c2f_off, *c2f;        // cell -> faces (ascending)
    const int32_t* c2fs;                 // as c2f, ~face where the cell is the face's neighbour (the gathers' sign)
    const int32_t *c2c_off, *c2c;        // cell -> face neighbours (sorted)
    // Gradient stencil in warp slices: cells 32s..32s+31 form slice s; its
    // entries occupy slots [g_soff[s], g_soff[s+1]) with entry k of the cell
    // in lane l at slot g_soff[s] + 32 k + l, each cell's entries in stencil
    // order and padded to the slice's longest stencil with (own cell, zero
    // weights), so a warp reads every entry array coalesced.
    const int64_t* g_soff;               // ceil(n/32) + 1
    const int32_t* g_col;                // slots
    const double *g_wx, *g_wy, *g_wz;    // LSQ coefficients per slot
    const BcPatch* patches;
    int32_t n_patches;
    const double* wall_dist;             // n (SA)
    // linear-system row of each cell (n) when the BSR matrix and its vectors
    // are stored in colour order; null: row = cell
    const int32_t* row_of;
};

__host__ __device__ inline int32_t row_index(const DevMesh& m, int32_t c) { return m.row_of ? m.row_of[c] : c; }

struct GasParams {
    double gamma, R, cv, cp, prandtl, prandtl_turb;
};

// Mutable per-cell/face fields (SoA).  Variable v of q lives at q + v*nt,
// gradient plane p of variable v at grad + (v*3+p)*nt.
struct DevFields {
    double* U;       // nv * n
    double* q;       // 5 * nt
    double* grad;    // nv_grad * 3 * nt
    double* phi;     // 5 * n
    double* fflux;   // 6 * nf, face-major: the 5 face fluxes then A*s_max of face f at fflux + 6 f
    double* res;     // nv * n
    double* lam;     // n
    double* dt;      // n
    double* alpha;   // n
    // Spalart-Allmaras scratch
    double* nu;      // nt: specific nu_tilde
    double* rho;     // nt: density
    double* mut;     // nt: eddy viscosity
};

inline unsigned grid_for(int64_t threads, int block) {
    const int64_t g = (threads + block - 1) / block;
    return static_cast<unsigned>(g < 1 ? 1 : g);
}

}  // namespace cfdg
