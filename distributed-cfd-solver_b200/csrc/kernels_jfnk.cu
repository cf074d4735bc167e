// Jacobian-free Newton-Krylov product and step control.  The reference's
// BackwardEuler (include/cfd/solver/compressible/time/implicit_euler.hpp:34-76)
// solves with the assembled first-order matrix; here the Krylov product can
// instead be the directional derivative of the full second-order residual,
//   y = (V/dt) x + (R(U + eps x) - R(U)) / eps,
// with the assembled matrix kept as the SGS preconditioner.  One step length
// eps serves the whole direction: no conserved variable moves by more than
// eps_rel of its RMS (the variables differ by orders of magnitude in SI
// units, rho nu~ is ~1e-5 of rho E).
//
// Layouts: U, R (and the perturbed copies) are SoA in cell order
// (U[v*n + c]); Krylov vectors are AoS in linear-system row order
// (x[row*NV + v], row = row_of[c] on a colour-ordered system).  Every
// kernel walks cells, so the SoA planes are read coalesced and each row's
// NV contiguous entries are one 40/48-byte access.
//
// Reductions are per block in a fixed order followed by a single-block
// finaliser over the partials in block order: the grid depends only on the
// problem size, so results repeat run to run.
#include "kernels.hpp"
#include "krylov.hpp"

namespace cfdg {

namespace {

constexpr int kJfThreads = 256;
constexpr int64_t kJfGridCap = 148 * 8;

inline unsigned jf_grid(int64_t items) {
    const int64_t g = grid_for(items, kJfThreads);
    return static_cast<unsigned>(g < kJfGridCap ? g : kJfGridCap);
}

// Block maximum of K values (all non-negative); thread 0 stores them.
template <int K>
__device__ __forceinline__ void block_max_store(double (&val)[K], double* __restrict__ out) {
    __shared__ double sh[K][kJfThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double x = val[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_down_sync(0xffffffffu, x, o));
        if (lane == 0) sh[k][warp] = x;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double x = (lane < kJfThreads / 32) ? sh[k][lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x = fmax(x, __shfl_down_sync(0xffffffffu, x, o));
            if (lane == 0) out[k] = x;
        }
    }
}

// Per-block sums of U_v^2 (RMS of each conserved variable).
template <int NV>
__global__ void __launch_bounds__(kJfThreads) k_jf_sumsq(int32_t n, const double* __restrict__ U,
                                                         double* __restrict__ partials) {
    double s[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] = 0.0;
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const double u = U[int64_t(v) * n + c];
            s[v] += u * u;
        }
    block_reduce_store<NV, kJfThreads>(s, partials + size_t(blockIdx.x) * NV);
}

// scal[v] = sqrt(mean U_v^2) + 1e-300: one block sums each variable's
// partials (thread t: blocks t, t+T, ..., then the fixed-order tree).
template <int NV>
__global__ void __launch_bounds__(kJfThreads) k_jf_rms_fin(int nblocks, int32_t n, const double* __restrict__ partials,
                                                           double* __restrict__ scal) {
    __shared__ double tot[NV];
    double s[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
        for (int v = 0; v < NV; ++v) s[v] += partials[size_t(b) * NV + v];
    block_reduce_store<NV, kJfThreads>(s, tot);
    __syncthreads();
    if (threadIdx.x < NV) scal[threadIdx.x] = sqrt(tot[threadIdx.x] / double(n)) + 1e-300;
}

// Per-block max |x_v| over the rows (x: AoS rows of NV).
template <int NV>
__global__ void __launch_bounds__(kJfThreads) k_jf_vmax(int32_t rows, const double* __restrict__ x,
                                                        double* __restrict__ partials, const int* __restrict__ active) {
    if (active && *active != 0) return;
    double m[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) m[v] = 0.0;
    for (int32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x)
#pragma unroll
        for (int v = 0; v < NV; ++v) m[v] = fmax(m[v], fabs(x[int64_t(r) * NV + v]));
    block_max_store<NV>(m, partials + size_t(blockIdx.x) * NV);
}

// eps = eps_rel / max_v(max|x_v| / rms(U_v)), 0 for x = 0 (scal[kJfEps]).
template <int NV>
__global__ void __launch_bounds__(kJfThreads) k_jf_eps(int nblocks, const double* __restrict__ partials,
                                                       double* __restrict__ scal, double eps_rel,
                                                       const int* __restrict__ active) {
    if (active && *active != 0) return;
    __shared__ double mx[NV];
    double m[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) m[v] = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
        for (int v = 0; v < NV; ++v) m[v] = fmax(m[v], partials[size_t(b) * NV + v]);
    block_max_store<NV>(m, mx);
    __syncthreads();
    if (threadIdx.x != 0) return;
    double w = 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) w = fmax(w, mx[v] / scal[v]);
    scal[kJfEps] = (w > 0.0 && isfinite(w)) ? eps_rel / w : 0.0;
}

// Up = U + eps x (x in row order).
template <int NV>
__global__ void __launch_bounds__(kJfThreads) k_jf_perturb(DevMesh m, const double* __restrict__ U,
                                                           const double* __restrict__ x,
                                                           const double* __restrict__ scal, double* __restrict__ Up,
                                                           const int* __restrict__ active) {
    if (active && *active != 0) return;
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.n) return;
    const double e = scal[kJfEps];
    const int64_t n = m.n, r = row_index(m, c);
#pragma unroll
    for (int v = 0; v < NV; ++v) Up[v * n + c] = U[v * n + c] + e * x[r * NV + v];
}

// y = (alpha - V diag) x + (R(U + eps x) + b) / eps, b = -R(U); dots of the
// result as the SpMV computes them (DotSpec; null operands stand for y).
// alpha - V diag is V/dt of the pseudo-time step alone: the BDF term of an
// unsteady residual is inside R and its derivative inside the difference.
template <int NV, int ND>
__global__ void __launch_bounds__(kJfThreads) k_jf_combine(DevMesh m, const double* __restrict__ alpha, double diag,
                                                           const double* __restrict__ x, const double* __restrict__ b,
                                                           const double* __restrict__ resp,
                                                           const double* __restrict__ scal, double* __restrict__ y,
                                                           DotSpec ds, double* __restrict__ partials,
                                                           const int* __restrict__ active) {
    if (active && *active != 0) return;
    const double e = scal[kJfEps];
    const int64_t n = m.n;
    double pr[ND > 0 ? ND : 1];
#pragma unroll
    for (int k = 0; k < (ND > 0 ? ND : 1); ++k) pr[k] = 0.0;
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < m.n; c += gridDim.x * blockDim.x) {
        const int64_t r = row_index(m, c);
        const double ap = alpha[c] - m.vol[c] * diag;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const int64_t t = r * NV + v;
            const double xv = x[t];
            const double yv = e > 0.0 ? ap * xv + (resp[v * n + c] + b[t]) / e : ap * xv;
            y[t] = yv;
            if constexpr (ND > 0) {
#pragma unroll
                for (int k = 0; k < ND; ++k) {
                    const double a = ds.a[k] ? ds.a[k][t] : yv;
                    const double bb = ds.b[k] ? ds.b[k][t] : yv;
                    pr[k] += a * bb;
                }
            }
        }
    }
    if constexpr (ND > 0) block_reduce_store<ND, kJfThreads>(pr, partials + size_t(blockIdx.x) * ND);
}

// Largest relative change of the update per block: |du_rho / rho|,
// |du_E / E| and, with the turbulence variable, |du_nu| / (|rho nu~| +
// 1e-3 rms(rho nu~)).
template <int NV>
__global__ void __launch_bounds__(kJfThreads) k_jf_step_ratio(DevMesh m, const double* __restrict__ U,
                                                              const double* __restrict__ du,
                                                              const double* __restrict__ scal,
                                                              double* __restrict__ partials) {
    double w[1] = {0.0};
    const int64_t n = m.n;
    const double floor_nu = NV == 6 ? 1e-3 * scal[5] : 0.0;
    for (int32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < m.n; c += gridDim.x * blockDim.x) {
        const int64_t r = row_index(m, c);
        w[0] = fmax(w[0], fabs(du[r * NV + 0] / U[c]));
        w[0] = fmax(w[0], fabs(du[r * NV + 4] / U[4 * n + c]));
        if constexpr (NV == 6) w[0] = fmax(w[0], fabs(du[r * NV + 5]) / (fabs(U[5 * n + c]) + floor_nu));
    }
    block_max_store<1>(w, partials + blockIdx.x);
}

// scal[kJfStep] = min(1, max_change / worst).
__global__ void __launch_bounds__(kJfThreads) k_jf_step_fin(int nblocks, const double* __restrict__ partials,
                                                            double max_change, double* __restrict__ scal) {
    __shared__ double mx[1];
    double w[1] = {0.0};
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) w[0] = fmax(w[0], partials[b]);
    block_max_store<1>(w, mx);
    __syncthreads();
    if (threadIdx.x == 0) scal[kJfStep] = (mx[0] > max_change) ? max_change / mx[0] : 1.0;
}

}  // namespace

int jf_partial_blocks(int32_t n) { return static_cast<int>(jf_grid(n)); }

void launch_jf_rms(int32_t n, int nv, const double* U, double* partials, double* scal, cudaStream_t s) {
    const unsigned gr = jf_grid(n);
    if (nv == 6) k_jf_sumsq<6><<<gr, kJfThreads, 0, s>>>(n, U, partials);
    else k_jf_sumsq<5><<<gr, kJfThreads, 0, s>>>(n, U, partials);
    if (nv == 6) k_jf_rms_fin<6><<<1, kJfThreads, 0, s>>>(static_cast<int>(gr), n, partials, scal);
    else k_jf_rms_fin<5><<<1, kJfThreads, 0, s>>>(static_cast<int>(gr), n, partials, scal);
}

void launch_jf_eps(int32_t rows, int nv, const double* x, double* partials, double* scal, double eps_rel,
                   const int* active, cudaStream_t s) {
    const unsigned gr = jf_grid(rows);
    if (nv == 6) k_jf_vmax<6><<<gr, kJfThreads, 0, s>>>(rows, x, partials, active);
    else k_jf_vmax<5><<<gr, kJfThreads, 0, s>>>(rows, x, partials, active);
    if (nv == 6) k_jf_eps<6><<<1, kJfThreads, 0, s>>>(static_cast<int>(gr), partials, scal, eps_rel, active);
    else k_jf_eps<5><<<1, kJfThreads, 0, s>>>(static_cast<int>(gr), partials, scal, eps_rel, active);
}

void launch_jf_perturb(const DevMesh& m, int nv, const double* U, const double* x, const double* scal, double* Up,
                       const int* active, cudaStream_t s) {
    const unsigned gr = grid_for(m.n, kJfThreads);
    if (nv == 6) k_jf_perturb<6><<<gr, kJfThreads, 0, s>>>(m, U, x, scal, Up, active);
    else k_jf_perturb<5><<<gr, kJfThreads, 0, s>>>(m, U, x, scal, Up, active);
}

int launch_jf_combine(const DevMesh& m, int nv, const double* alpha, double diag, const double* x, const double* b,
                      const double* resp, const double* scal, double* y, const DotSpec& ds, double* partials,
                      const int* active, cudaStream_t s) {
    const unsigned gr = jf_grid(m.n);
#define CFDG_JFC(NV, ND) \
    k_jf_combine<NV, ND><<<gr, kJfThreads, 0, s>>>(m, alpha, diag, x, b, resp, scal, y, ds, partials, active)
    if (nv == 6) {
        if (ds.n == 0) CFDG_JFC(6, 0);
        else if (ds.n == 1) CFDG_JFC(6, 1);
        else CFDG_JFC(6, 5);
    } else {
        if (ds.n == 0) CFDG_JFC(5, 0);
        else if (ds.n == 1) CFDG_JFC(5, 1);
        else CFDG_JFC(5, 5);
    }
#undef CFDG_JFC
    return static_cast<int>(gr);
}

void launch_jf_step_scale(const DevMesh& m, int nv, const double* U, const double* du, double* partials, double* scal,
                          double max_change, cudaStream_t s) {
    const unsigned gr = jf_grid(m.n);
    if (nv == 6) k_jf_step_ratio<6><<<gr, kJfThreads, 0, s>>>(m, U, du, scal, partials);
    else k_jf_step_ratio<5><<<gr, kJfThreads, 0, s>>>(m, U, du, scal, partials);
    k_jf_step_fin<<<1, kJfThreads, 0, s>>>(static_cast<int>(gr), partials, max_change, scal);
}

}  // namespace cfdg
