// Inputs and training samples of the learned Newton initial guess.
//
// Per cell c and variable v, with e = (dt_c / V_c) * b (the explicit
// pseudo-time update, b = -R):
//   g1 = e / s_e, g2 = (U - U_inf) / s_U, g3 = dU_prev / s_d,
// where s_e and s_d are the RMS over cells of e and of the previous Newton
// update (one shared value for the momentum vector) and s_U a free-stream
// scale.  The 48 features are
//   [g1, g2, g3, mean_nb g1, mean_nb g3, max_nb g1, max_nb g2]
// (7 groups of nvars over the face neighbours, zero padded) and, last,
// log10(mean_v s_e / s_d) / 4 and log10(CFL) / 4, in bf16.  The network
// predicts dU / s_d: the update relative to the previous one, an O(1)
// quantity in every phase of the convergence.
#include <cuda_bf16.h>

#include <cmath>

#include "guess.hpp"
#include "kernels.hpp"
#include "mlp.hpp"

namespace cfdg {

namespace {

constexpr int kSumThreads = 256;

template <int NV>
__global__ void __launch_bounds__(kSumThreads) k_guess_sums(int32_t n, const int32_t* __restrict__ row_of,
                                                           const double* __restrict__ b,
                                                           const double* __restrict__ dt,
                                                           const double* __restrict__ vol,
                                                           const double* __restrict__ du_prev,
                                                           double* __restrict__ partials) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[2 * NV];
#pragma unroll
    for (int k = 0; k < 2 * NV; ++k) acc[k] = 0.0;
    if (c < n) {
        const double w = dt[c] / vol[c];
        const int64_t r = row_of ? row_of[c] : c;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const double e = w * b[r * NV + v];
            const double d = du_prev[r * NV + v];
            acc[v] = e * e;
            acc[NV + v] = d * d;
        }
    }
    block_reduce_store<2 * NV, kSumThreads>(acc, partials + size_t(blockIdx.x) * (2 * NV));
}

// gscale layout: [0,8) s_e, [8,16) s_d, [16,24) s_U, [24,32) U_inf.  The
// three momentum components share one scale (the RMS of the vector), so a
// component that stays at round-off (spanwise momentum of a quasi-2-D flow)
// is not blown up to O(1).
template <int NV>
__global__ void k_guess_scales(int32_t n, const double* __restrict__ partials, int nblocks, double* gscale) {
    __shared__ double sq[2 * NV];
    const int k = threadIdx.x;
    if (k < 2 * NV) {
        double s = 0.0;
        for (int i = 0; i < nblocks; ++i) s += partials[size_t(i) * (2 * NV) + k];
        sq[k] = s / double(n > 0 ? n : 1);
    }
    __syncthreads();
    if (k >= 2 * NV) return;
    const int grp = k / NV, v = k - grp * NV;
    double ms = sq[k];
    if (v >= 1 && v <= 3) ms = (sq[grp * NV + 1] + sq[grp * NV + 2] + sq[grp * NV + 3]) * (1.0 / 3.0);
    const double rms = sqrt(ms);
    gscale[grp * 8 + v] = (rms > 0.0 && isfinite(rms)) ? rms : 1.0;
}

__device__ __forceinline__ uint16_t bf(double x) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(static_cast<float>(x)));
}

template <int NV>
__global__ void __launch_bounds__(128) k_guess_features(DevMesh m, const double* __restrict__ U,
                                                       const double* __restrict__ b, const double* __restrict__ dt,
                                                       const double* __restrict__ du_prev,
                                                       const double* __restrict__ gscale, double lcfl,
                                                       uint16_t* __restrict__ feat) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.n) return;
    const int64_t n = m.n;
    double ise[NV], isd[NV], isu[NV], uinf[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        ise[v] = 1.0 / gscale[v];
        isd[v] = 1.0 / gscale[8 + v];
        isu[v] = 1.0 / gscale[16 + v];
        uinf[v] = gscale[24 + v];
    }
    auto groups = [&](int32_t k, double* g1, double* g2, double* g3) {
        const double w = dt[k] / m.vol[k];
        const int64_t r = row_index(m, k);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            g1[v] = w * b[r * NV + v] * ise[v];
            g2[v] = (U[v * n + k] - uinf[v]) * isu[v];
            g3[v] = du_prev[r * NV + v] * isd[v];
        }
    };
    double f[kMlpIn];
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i) f[i] = 0.0;
    double s1[NV], s3[NV], mx1[NV], mx2[NV];
    groups(c, f, f + NV, f + 2 * NV);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        s1[v] = s3[v] = 0.0;
        mx1[v] = mx2[v] = -1.0e300;
    }
    const int32_t j0 = m.c2c_off[c], j1 = m.c2c_off[c + 1];
    for (int32_t j = j0; j < j1; ++j) {
        double g1[NV], g2[NV], g3[NV];
        groups(m.c2c[j], g1, g2, g3);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            s1[v] += g1[v];
            s3[v] += g3[v];
            mx1[v] = fmax(mx1[v], g1[v]);
            mx2[v] = fmax(mx2[v], g2[v]);
        }
    }
    const double inv = (j1 > j0) ? 1.0 / double(j1 - j0) : 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        f[3 * NV + v] = s1[v] * inv;
        f[4 * NV + v] = s3[v] * inv;
        f[5 * NV + v] = (j1 > j0) ? mx1[v] : 0.0;
        f[6 * NV + v] = (j1 > j0) ? mx2[v] : 0.0;
    }
    double ratio = 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) ratio += gscale[v] * isd[v];
    f[kMlpIn - 2] = 0.25 * log10(fmax(ratio / NV, 1e-30));
    f[kMlpIn - 1] = lcfl;
    uint32_t packed[kMlpIn / 2];
#pragma unroll
    for (int i = 0; i < kMlpIn / 2; ++i) packed[i] = uint32_t(bf(f[2 * i])) | (uint32_t(bf(f[2 * i + 1])) << 16);
    // the feature row of a cell is its linear-system row, so that the
    // network's outputs land in the layout of the Krylov vectors
    uint4* dst = reinterpret_cast<uint4*>(feat + int64_t(row_index(m, c)) * kMlpIn);
#pragma unroll
    for (int q = 0; q < kMlpIn / 8; ++q)
        dst[q] = make_uint4(packed[4 * q], packed[4 * q + 1], packed[4 * q + 2], packed[4 * q + 3]);
}

// Samples c = phase + k * stride: features row and target dU / s_d.
__global__ void k_guess_append(int32_t n, const int32_t* __restrict__ row_of, int nv, int32_t stride, int32_t phase,
                               int64_t count, const uint16_t* __restrict__ feat, const double* __restrict__ du,
                               const double* __restrict__ gscale, uint16_t* __restrict__ X, float* __restrict__ T) {
    const int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= count) return;
    const int64_t c0 = phase + k * stride;
    const int64_t c = row_of ? row_of[c0] : c0;
    const uint4* src = reinterpret_cast<const uint4*>(feat + c * kMlpIn);
    uint4* dst = reinterpret_cast<uint4*>(X + k * kMlpIn);
#pragma unroll
    for (int q = 0; q < kMlpIn / 8; ++q) dst[q] = src[q];
    for (int v = 0; v < kMlpOut; ++v)
        T[k * kMlpOut + v] = (v < nv) ? static_cast<float>(du[c * nv + v] / gscale[8 + v]) : 0.0f;
}

}  // namespace

int guess_sum_blocks(int32_t n) { return static_cast<int>((int64_t(n) + kSumThreads - 1) / kSumThreads); }

void launch_guess_scales(int32_t n, const int32_t* row_of, int nv, const double* b, const double* dt,
                         const double* vol, const double* du_prev, double* partials, double* gscale, cudaStream_t s) {
    const int nb = guess_sum_blocks(n);
    if (nv == 6) {
        k_guess_sums<6><<<nb, kSumThreads, 0, s>>>(n, row_of, b, dt, vol, du_prev, partials);
        k_guess_scales<6><<<1, 32, 0, s>>>(n, partials, nb, gscale);
    } else {
        k_guess_sums<5><<<nb, kSumThreads, 0, s>>>(n, row_of, b, dt, vol, du_prev, partials);
        k_guess_scales<5><<<1, 32, 0, s>>>(n, partials, nb, gscale);
    }
}

void launch_guess_features(const DevMesh& m, int nv, const double* U, const double* b, const double* dt,
                           const double* du_prev, const double* gscale, double cfl, uint16_t* feat, cudaStream_t s) {
    const unsigned gr = grid_for(m.n, 128);
    const double lcfl = 0.25 * std::log10(cfl > 0.0 ? cfl : 1.0);
    if (nv == 6) k_guess_features<6><<<gr, 128, 0, s>>>(m, U, b, dt, du_prev, gscale, lcfl, feat);
    else k_guess_features<5><<<gr, 128, 0, s>>>(m, U, b, dt, du_prev, gscale, lcfl, feat);
}

void launch_guess_append(int32_t n, const int32_t* row_of, int nv, int32_t stride, int32_t phase, int64_t count,
                         const uint16_t* feat, const double* du, const double* gscale, uint16_t* X, float* T,
                         cudaStream_t s) {
    if (count <= 0) return;
    k_guess_append<<<grid_for(count, 128), 128, 0, s>>>(n, row_of, nv, stride, phase, count, feat, du, gscale, X, T);
}

}  // namespace cfdg
