// Kernel launchers (host declarations) and device reduction helpers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_common.cuh"

namespace cfdg {

#ifdef __CUDACC__
// Deterministic block reduction of K values: warp shuffle trees, then the
// warps' results summed in warp order by warp 0.  Thread 0 stores K values.
template <int K, int BLOCK>
__device__ __forceinline__ void block_reduce_store(double (&val)[K], double* __restrict__ out) {
    __shared__ double sh[K][BLOCK / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double x = val[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) sh[k][warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double x = (lane < BLOCK / 32) ? sh[k][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) out[k] = x;
        }
    }
}
#endif

// ---------------------------------------------------------------- residual
void launch_primitives(const DevMesh& m, const DevFields& f, const GasParams& g, cudaStream_t s);
void launch_gradient(const DevMesh& m, const double* src, double* dst, int nvars, cudaStream_t s);
void launch_limiter_ghostgrad(const DevMesh& m, const DevFields& f, const GasParams& g, bool limit, int limiter,
                              double venkat_k, cudaStream_t s);
void launch_face_flux(const DevMesh& m, const DevFields& f, const GasParams& g, bool muscl, bool visc,
                      cudaStream_t s);
void launch_cell_residual(const DevMesh& m, const DevFields& f, cudaStream_t s);
int norm_blocks(int32_t n);
void launch_norms(int32_t n, int nv, const double* res, double* partials, double* l2, cudaStream_t s);
void launch_dt_rhs(const DevMesh& m, const DevFields& f, int nv, double cfl, double diag, double* b, cudaStream_t s);
void launch_unsteady_source(int32_t n, int nv, const double* vol, const double* U, const double* Un,
                            const double* Unm1, double c0, double c1, double c2, double* res, cudaStream_t s);
void launch_state_update(const DevMesh& m, double* U, const double* du, int nv, const double* scale, cudaStream_t s);
void launch_fill(double* x, int64_t count, double value, cudaStream_t s);

// -------------------------------------------------------- Spalart-Allmaras
struct SaParams {
    double nu_inf;      // freestream specific nu_tilde
    double sigma, cb1, cb2, kappa, cw1, cw2, cw3, cv1;
};
void launch_sa_pre(const DevMesh& m, const DevFields& f, const GasParams& g, const SaParams& sa, double* rhonu_g,
                   cudaStream_t s);
void launch_output_fields(int32_t n, int nv, const double* U, const GasParams& g, double cv1, double* out,
                          cudaStream_t s);
void launch_sa_sweep(const DevMesh& m, const DevFields& f, const GasParams& g, const SaParams& sa,
                     const double* rhonu_g, const double* gnu, double* face, double* jac, double* dsrc,
                     cudaStream_t s);

// ---------------------------------------------------------------- Jacobian
struct JacStructure {
    const int32_t* row_ptr;   // n+1
    const int32_t* cols;      // nnzb
    const int32_t* diag;      // n
    const int32_t* face_pos;  // 2*ni: block (owner,neigh), block (neigh,owner)
    bool full_viscous;        // thin-layer operator with the normal-stress term + no-slip ghost
    // Spalart-Allmaras (6x6 blocks): per face the pair d(nu_tilde flux)/d(rho
    // nu_tilde) of owner and neighbour at [2f, 2f+1], and the destruction
    // derivative per cell; null without the model
    const double* sa_jac;
    const double* sa_dsrc;
    const int32_t* cell_of;   // cell of each block row (colour-ordered system); null: row = cell
};
template <typename MT>
void launch_jacobian(const DevMesh& m, const DevFields& f, const GasParams& g, const JacStructure& js, int bs,
                     bool visc, MT* values, cudaStream_t s);


// ------------------------------------------- Jacobian-free Newton-Krylov
// Device scalars of the Jacobian-free product (a buffer of kJfScalars
// doubles): [0, nv) RMS of each conserved variable, then the product's step
// length and the Newton step's relaxation factor.
enum : int { kJfEps = 6, kJfStep = 7, kJfScalars = 16 };
int jf_partial_blocks(int32_t n);  // partial rows of the reductions below (x nv doubles)
void launch_jf_rms(int32_t n, int nv, const double* U, double* partials, double* scal, cudaStream_t s);
void launch_jf_eps(int32_t rows, int nv, const double* x, double* partials, double* scal, double eps_rel,
                   const int* active, cudaStream_t s);
void launch_jf_perturb(const DevMesh& m, int nv, const double* U, const double* x, const double* scal, double* Up,
                       const int* active, cudaStream_t s);
void launch_jf_step_scale(const DevMesh& m, int nv, const double* U, const double* du, double* partials, double* scal,
                          double max_change, cudaStream_t s);

// ------------------------------------------------------ restarted GMRES
// Basis V: vectors k at V + k*ld.  h[k0 + k] = V_{k0+k} . w for k < kn
// (partials: gm_partial_blocks(len) * gm_chunk() doubles); w -= sum h_k V_k
// (subtract) or w = sum h_k V_k; y = a x (+ y).
int gm_partial_blocks(int64_t len);
int gm_chunk();
void launch_gm_dots(int64_t len, const double* V, int64_t ld, int k0, int kn, const double* w, double* partials,
                    double* h, cudaStream_t s);
void launch_gm_update(int64_t len, const double* V, int64_t ld, int kn, const double* h, double* w, bool subtract,
                      cudaStream_t s);
void launch_gm_axpy(int64_t len, double a, const double* x, double* y, bool accumulate, cudaStream_t s);

// ------------------------------------------------------------ linear algebra
struct BsrView {
    int32_t n, bs;
    const int32_t* row_ptr;
    const int32_t* cols;
    const int32_t* diag;
};
// inverse: store D^-1 instead of the pivoted LU factors (multicolour sweep)
template <typename MT>
void launch_lu_setup(const BsrView& A, const MT* vals, MT* lu, int8_t* piv, int* err_flag, bool inverse,
                     cudaStream_t s);
int spmv_blocks(int32_t n, int32_t bs);
int dot_blocks(int64_t len);

}  // namespace cfdg
