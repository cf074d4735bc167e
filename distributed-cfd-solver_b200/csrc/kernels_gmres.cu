// Restarted GMRES building blocks (right-preconditioned, classical
// Gram-Schmidt with one reorthogonalisation pass).  The Krylov basis is one
// array of (restart + 1) vectors of `len` doubles; the projections go
// through fused multi-dot products (up to kGmChunk basis vectors against w
// per launch, w read once per chunk) and one fused update
// w -= sum_k h_k V_k.  Reductions are per block in a fixed order, then a
// finaliser per coefficient over the blocks in block order: the grid depends
// only on the length, so the coefficients repeat run to run.
#include "kernels.hpp"

namespace cfdg {

namespace {

constexpr int kGmThreads = 256;
constexpr int64_t kGmGridCap = 148 * 8;
constexpr int kGmChunk = 8;

inline unsigned gm_grid(int64_t len) {
    const int64_t g = grid_for(len, kGmThreads);
    return static_cast<unsigned>(g < kGmGridCap ? g : kGmGridCap);
}

// partials[b * kGmChunk + k] = sum over block b's entries of V_{k0+k} . w,
// k < kn (kn <= kGmChunk).  V = w with kn = 1 gives |w|^2.
__global__ void __launch_bounds__(kGmThreads) k_gm_dots(int64_t len, const double* __restrict__ V, int64_t ld, int k0,
                                                        int kn, const double* __restrict__ w,
                                                        double* __restrict__ partials) {
    double s[kGmChunk];
#pragma unroll
    for (int k = 0; k < kGmChunk; ++k) s[k] = 0.0;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < len; t += int64_t(gridDim.x) * blockDim.x) {
        const double wt = w[t];
#pragma unroll
        for (int k = 0; k < kGmChunk; ++k)
            if (k < kn) s[k] += V[int64_t(k0 + k) * ld + t] * wt;
    }
    block_reduce_store<kGmChunk, kGmThreads>(s, partials + size_t(blockIdx.x) * kGmChunk);
}

// h[k0 + k] = sum over blocks of partials[b * kGmChunk + k], one warp per
// coefficient: lane-strided sums in block order, then a fixed shuffle tree.
__global__ void k_gm_dots_fin(int nblocks, int k0, int kn, const double* __restrict__ partials,
                              double* __restrict__ h) {
    const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (k >= kn) return;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += partials[size_t(b) * kGmChunk + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) h[k0 + k] = s;
}

// w -= sum_{k < kn} h_k V_k  (sign = -1), or w = sum_{k < kn} h_k V_k
// (sign = 0: the combination of the basis with the least-squares solution).
__global__ void __launch_bounds__(kGmThreads) k_gm_update(int64_t len, const double* __restrict__ V, int64_t ld, int kn,
                                                          const double* __restrict__ h, double* __restrict__ w,
                                                          int sign) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < len; t += int64_t(gridDim.x) * blockDim.x) {
        double acc = sign ? w[t] : 0.0;
        for (int k = 0; k < kn; ++k) {
            const double c = h[k];
            acc = sign ? acc - c * V[int64_t(k) * ld + t] : acc + c * V[int64_t(k) * ld + t];
        }
        w[t] = acc;
    }
}

// y = a x (+ y when accumulate)
__global__ void __launch_bounds__(kGmThreads) k_gm_axpy(int64_t len, double a, const double* __restrict__ x,
                                                        double* __restrict__ y, int accumulate) {
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < len; t += int64_t(gridDim.x) * blockDim.x)
        y[t] = accumulate ? y[t] + a * x[t] : a * x[t];
}

}  // namespace

int gm_partial_blocks(int64_t len) { return static_cast<int>(gm_grid(len)); }
int gm_chunk() { return kGmChunk; }

void launch_gm_dots(int64_t len, const double* V, int64_t ld, int k0, int kn, const double* w, double* partials,
                    double* h, cudaStream_t s) {
    const unsigned gr = gm_grid(len);
    for (int c = 0; c < kn; c += kGmChunk) {
        const int m = kn - c < kGmChunk ? kn - c : kGmChunk;
        k_gm_dots<<<gr, kGmThreads, 0, s>>>(len, V, ld, k0 + c, m, w, partials);
        k_gm_dots_fin<<<1, 32 * kGmChunk, 0, s>>>(static_cast<int>(gr), k0 + c, m, partials, h);
    }
}

void launch_gm_update(int64_t len, const double* V, int64_t ld, int kn, const double* h, double* w, bool subtract,
                      cudaStream_t s) {
    k_gm_update<<<gm_grid(len), kGmThreads, 0, s>>>(len, V, ld, kn, h, w, subtract ? 1 : 0);
}

void launch_gm_axpy(int64_t len, double a, const double* x, double* y, bool accumulate, cudaStream_t s) {
    k_gm_axpy<<<gm_grid(len), kGmThreads, 0, s>>>(len, a, x, y, accumulate ? 1 : 0);
}

}  // namespace cfdg
