// Per-cell MLP of the learned Newton initial guess on the 5th-generation
// tensor cores: one elected thread issues tcgen05.mma on BF16 operands
// staged in shared memory (K-major core-matrix tiles), the FP32
// accumulators live in tensor memory and return to registers through
// tcgen05.ld for the bias / ReLU / loss epilogues.
//
// Forward (inference and training): 128 cells per tile,
//   Z1 = X W1^T + b1, H1 = relu(Z1), Z2 = H1 W2^T + b2, H2 = relu(Z2),
//   Y = H2 W3^T + b3.
// Backward (training), all products on the tensor cores with M = 128:
//   dY = Y - T (masked to the used outputs), dH2 = dY W3, dZ2 = dH2 * [Z2>0],
//   dH1 = dZ2 W2, dZ1 = dH1 * [Z1>0], and the weight gradients
//   dW3^T = H2^T dY, dW2 = dZ2^T H1, dW1 = dZ1^T X accumulated over the
//   CTA's tiles in tensor memory; a ones row appended to the second operand
//   yields the bias gradients in the same products.
#include <cuda_bf16.h>

#include <algorithm>

#include "mlp.hpp"
#include "tcgen05.cuh"

namespace cfdg {

namespace {

constexpr uint32_t kWaitLimit = 1u << 26;  // mbarrier polls before a wait gives up

__device__ __forceinline__ uint16_t f2bf(float x) { return __bfloat16_as_ushort(__float2bfloat16_rn(x)); }

// Row-major bf16 [R x K] (global) -> K-major core tile; rows >= valid are zero.
__device__ void load_tile(uint8_t* tile, const uint16_t* __restrict__ g, int R, int K, int64_t valid) {
    const int kc = K >> 3;
    for (int q = threadIdx.x; q < R * kc; q += blockDim.x) {
        const int r = q / kc, c = q - r * kc;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (r < valid) v = *reinterpret_cast<const uint4*>(g + int64_t(r) * K + c * 8);
        *reinterpret_cast<uint4*>(tile + tc::core_offset(r, c * 8, K)) = v;
    }
}

// Transposed load: tile element (r, k) = g[k * R + r] (g row-major [K x R]).
__device__ void load_tile_t(uint8_t* tile, const uint16_t* __restrict__ g, int R, int K) {
    for (int q = threadIdx.x; q < R * K; q += blockDim.x) {
        const int r = q / K, k = q - r * K;
        *reinterpret_cast<uint16_t*>(tile + tc::core_offset(r, k, K)) = g[int64_t(k) * R + r];
    }
}

__device__ void zero_bytes(uint8_t* p, int bytes) {
    for (int q = threadIdx.x; q < bytes / 16; q += blockDim.x)
        reinterpret_cast<uint4*>(p)[q] = make_uint4(0u, 0u, 0u, 0u);
}

// Stores 8 consecutive bf16 values of row r (columns k..k+7) into a core tile.
__device__ __forceinline__ void store8(uint8_t* tile, int r, int k, int K, const float* v) {
    uint4 u;
    u.x = uint32_t(f2bf(v[0])) | (uint32_t(f2bf(v[1])) << 16);
    u.y = uint32_t(f2bf(v[2])) | (uint32_t(f2bf(v[3])) << 16);
    u.z = uint32_t(f2bf(v[4])) | (uint32_t(f2bf(v[5])) << 16);
    u.w = uint32_t(f2bf(v[6])) | (uint32_t(f2bf(v[7])) << 16);
    *reinterpret_cast<uint4*>(tile + tc::core_offset(r, k, K)) = u;
}

// Issues the K/16 MMAs of D[128 x N] (+)= A[128 x K] B[N x K]^T.
__device__ __forceinline__ void issue_gemm(uint32_t d_tmem, const uint8_t* a, const uint8_t* b, int N, int K,
                                          bool accumulate) {
    const uint32_t sbo = static_cast<uint32_t>(K >> 3) * 128u;
    const uint32_t id = tc::idesc_bf16_f32(128, N);
    const uint32_t sa = tc::smem_u32(a), sb = tc::smem_u32(b);
    for (int ks = 0; ks < K / 16; ++ks) {
        const uint64_t da = tc::smem_desc(sa + ks * 256u, 128u, sbo);
        const uint64_t db = tc::smem_desc(sb + ks * 256u, 128u, sbo);
        tc::mma_bf16(d_tmem, da, db, id, accumulate || ks > 0);
    }
}

// Waits for the commit of the current phase; the outcome is made uniform
// across the block.  On a timeout thread 0 records it in *err.
__device__ __forceinline__ bool wait_all(uint64_t* bar, uint32_t& phase, int* err) {
    bool ok = tc::mbar_wait(bar, phase, kWaitLimit);
    ok = __syncthreads_and(ok) != 0;
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
    phase ^= 1u;
    tc::fence_after_sync();
    return ok;
}

// Makes generic-proxy shared stores and completed TMEM loads visible
// before the next MMA issue.
__device__ __forceinline__ void to_mma() {
    tc::fence_before_sync();
    tc::fence_async_smem();
    __syncthreads();
    tc::fence_after_sync();
}

__device__ __forceinline__ uint32_t lane_base(uint32_t tbase) {
    return tbase + (static_cast<uint32_t>((threadIdx.x >> 5) * 32) << 16);
}

// On a failed wait: give the MMAs in flight a bounded time to finish, then
// release the tensor memory.
__device__ void abort_tc(uint64_t* bar, uint32_t phase, uint32_t tbase, uint32_t ncols) {
    tc::mbar_wait(bar, phase ^ 1u, kWaitLimit);
    tc::fence_before_sync();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tbase, ncols);
    }
}

// --------------------------------------------------------------- self-test
__global__ void __launch_bounds__(128) k_tc_selftest(const uint16_t* A, const uint16_t* B, float* D, int N, int K,
                                                     int* err) {
    extern __shared__ __align__(128) uint8_t smem[];
    uint8_t* sA = smem;                   // 128 x K
    uint8_t* sB = sA + 128 * K * 2;       // N x K
    uint64_t* bar = reinterpret_cast<uint64_t*>(sB + 64 * K * 2);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    load_tile(sA, A, 128, K, 128);
    load_tile(sB, B, N, K, N);
    if (threadIdx.x == 0) {
        tc::mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if ((threadIdx.x >> 5) == 0) {
        tc::tmem_alloc(slot, 128);
        tc::tmem_relinquish();
    }
    to_mma();
    const uint32_t tbase = *slot;
    uint32_t phase = 0;
    if (threadIdx.x == 0) {
        issue_gemm(tbase, sA, sB, N, K, false);
        tc::mma_commit(bar);
    }
    if (!wait_all(bar, phase, err)) {
        abort_tc(bar, phase, tbase, 128);
        return;
    }
    const int r = threadIdx.x;
    for (int c = 0; c < N; c += 16) {
        float v[16];
        tc::tmem_ld16(lane_base(tbase) + c, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) D[r * N + c + i] = v[i];
    }
    tc::fence_before_sync();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tbase, 128);
    }
}

// ------------------------------------------------------------ shared setup
struct FwdSmem {
    uint8_t *w1, *w2, *w3, *x, *h;
    float* bias;  // b1[64] b2[64] b3[16]
    uint64_t* bar;
    uint32_t* slot;
};
constexpr int kFwdSmem = 6144 + 8192 + 2048 + 12288 + 16384 + 144 * 4 + 16;

__device__ FwdSmem carve_fwd(uint8_t* smem) {
    FwdSmem s;
    s.w1 = smem;
    s.w2 = s.w1 + 6144;
    s.w3 = s.w2 + 8192;
    s.x = s.w3 + 2048;
    s.h = s.x + 12288;
    s.bias = reinterpret_cast<float*>(s.h + 16384);
    s.bar = reinterpret_cast<uint64_t*>(s.bias + 144);
    s.slot = reinterpret_cast<uint32_t*>(s.bar + 1);
    return s;
}

__device__ void load_net(const MlpDev& net, uint8_t* w1, uint8_t* w2, uint8_t* w3, float* bias) {
    load_tile(w1, net.w1, kMlpHid, kMlpIn, kMlpHid);
    load_tile(w2, net.w2, kMlpHid, kMlpHid, kMlpHid);
    load_tile(w3, net.w3, kMlpOut, kMlpHid, kMlpOut);
    for (int i = threadIdx.x; i < 144; i += blockDim.x) {
        float b;
        if (i < 64) b = net.params[kOffB1 + i];
        else if (i < 128) b = net.params[kOffB2 + i - 64];
        else b = net.params[kOffB3 + i - 128];
        bias[i] = b;
    }
}

// Hidden-layer epilogue: row r of acc (64 columns) + bias, ReLU, bf16 into
// the core tile `h`; returns the mask of positive pre-activations.
__device__ __forceinline__ uint64_t epi_hidden(uint32_t tacc, const float* bias, uint8_t* h) {
    const int r = threadIdx.x;
    uint64_t mask = 0;
#pragma unroll
    for (int c = 0; c < 64; c += 16) {
        float v[16];
        tc::tmem_ld16(lane_base(tacc) + c, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const float z = v[i] + bias[c + i];
            if (z > 0.0f) mask |= (uint64_t(1) << (c + i));
            v[i] = fmaxf(z, 0.0f);
        }
        store8(h, r, c, 64, v);
        store8(h, r, c + 8, 64, v + 8);
    }
    return mask;
}

// ----------------------------------------------------------- inference
__global__ void __launch_bounds__(128) k_mlp_forward(MlpDev net, const uint16_t* __restrict__ feat, int64_t rows,
                                                     const double* __restrict__ scale, int nv,
                                                     double* __restrict__ out, int* err) {
    extern __shared__ __align__(128) uint8_t smem[];
    const FwdSmem s = carve_fwd(smem);
    load_net(net, s.w1, s.w2, s.w3, s.bias);
    if (threadIdx.x == 0) {
        tc::mbar_init(s.bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if ((threadIdx.x >> 5) == 0) {
        tc::tmem_alloc(s.slot, 128);
        tc::tmem_relinquish();
    }
    to_mma();
    const uint32_t tbase = *s.slot;
    uint32_t phase = 0;
    const int r = threadIdx.x;
    double sc[kMlpOut];
#pragma unroll
    for (int v = 0; v < kMlpOut; ++v) sc[v] = (v < nv) ? scale[v] : 0.0;
    const int64_t ntiles = (rows + kMlpTile - 1) / kMlpTile;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t r0 = t * kMlpTile;
        load_tile(s.x, feat + r0 * kMlpIn, kMlpTile, kMlpIn, rows - r0);
        to_mma();
        if (threadIdx.x == 0) {
            issue_gemm(tbase, s.x, s.w1, 64, kMlpIn, false);
            tc::mma_commit(s.bar);
        }
        if (!wait_all(s.bar, phase, err)) return abort_tc(s.bar, phase, tbase, 128);
        epi_hidden(tbase, s.bias, s.h);
        to_mma();
        if (threadIdx.x == 0) {
            issue_gemm(tbase + 64, s.h, s.w2, 64, kMlpHid, false);
            tc::mma_commit(s.bar);
        }
        if (!wait_all(s.bar, phase, err)) return abort_tc(s.bar, phase, tbase, 128);
        epi_hidden(tbase + 64, s.bias + 64, s.h);
        to_mma();
        if (threadIdx.x == 0) {
            issue_gemm(tbase, s.h, s.w3, 16, kMlpHid, false);
            tc::mma_commit(s.bar);
        }
        if (!wait_all(s.bar, phase, err)) return abort_tc(s.bar, phase, tbase, 128);
        float y[16];
        tc::tmem_ld16(lane_base(tbase), y);
        if (r0 + r < rows) {
            double* o = out + (r0 + r) * nv;
            for (int v = 0; v < nv; ++v) o[v] = sc[v] * double(y[v] + s.bias[128 + v]);
        }
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
    }
    tc::fence_before_sync();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tbase, 128);
    }
}

// ------------------------------------------------------------- training
// Tensor-memory columns (512 allocated, one CTA per SM):
constexpr uint32_t kT1 = 0;      // Z1, then Y, then dH1   (64)
constexpr uint32_t kT2 = 64;     // Z2, then dH2           (64)
constexpr uint32_t kGW3 = 128;   // dW3^T rows=in, row 64 = db3 (16)
constexpr uint32_t kGW1 = 144;   // dW1 rows=out, col 48 = db1 (64)
constexpr uint32_t kGW2 = 208;   // dW2 rows=out, col 64 = db2 (80)

struct TrainSmem {
    uint8_t *w1, *w2, *w3, *w2t, *w3t, *x, *xt, *h, *h1t, *at, *dy, *dyt;
    float* bias;
    float* red;
    uint64_t* bar;
    uint32_t* slot;
};
constexpr int kTrainSmem = 6144 + 8192 + 2048 + 8192 + 2048 + 12288 + 16384 + 16384 + 20480 + 32768 + 4096 + 4096 +
                           144 * 4 + 128 * 4 + 16;

__device__ TrainSmem carve_train(uint8_t* smem) {
    TrainSmem s;
    s.w1 = smem;                 // W1   [64 x 48]
    s.w2 = s.w1 + 6144;          // W2   [64 x 64]
    s.w3 = s.w2 + 8192;          // W3   [16 x 64]
    s.w2t = s.w3 + 2048;         // W2^T [64 x 64]  (B of dH1 = dZ2 W2)
    s.w3t = s.w2t + 8192;        // W3^T [64 x 16]  (B of dH2 = dY W3)
    s.x = s.w3t + 2048;          // X    [128 x 48]
    s.xt = s.x + 12288;          // X^T  [64 x 128] (48 features, ones row 48, zeros)
    s.h = s.xt + 16384;          // H1 / H2 / dZ2 [128 x 64]
    s.h1t = s.h + 16384;         // H1^T [80 x 128] (ones row 64, zeros)
    s.at = s.h1t + 20480;        // H2^T / dZ2^T / dZ1^T [128 x 128] (row 64 ones, rows 65.. zero)
    s.dy = s.at + 32768;         // dY   [128 x 16]
    s.dyt = s.dy + 4096;         // dY^T [16 x 128]
    s.bias = reinterpret_cast<float*>(s.dyt + 4096);
    s.red = s.bias + 144;
    s.bar = reinterpret_cast<uint64_t*>(s.red + 128);
    s.slot = reinterpret_cast<uint32_t*>(s.bar + 1);
    return s;
}

__device__ __forceinline__ void put_bf16(uint8_t* tile, int r, int k, int K, float v) {
    *reinterpret_cast<uint16_t*>(tile + tc::core_offset(r, k, K)) = f2bf(v);
}

__global__ void __launch_bounds__(128, 1) k_mlp_grad(MlpDev net, const uint16_t* __restrict__ feat,
                                                     const float* __restrict__ target, int64_t rows,
                                                     float* __restrict__ partials, int* err) {
    extern __shared__ __align__(128) uint8_t smem[];
    const TrainSmem s = carve_train(smem);
    load_net(net, s.w1, s.w2, s.w3, s.bias);
    load_tile_t(s.w2t, net.w2, kMlpHid, kMlpHid);  // (in, out) = W2[out][in]
    load_tile_t(s.w3t, net.w3, kMlpHid, kMlpOut);  // (in, out) = W3[out][in]
    zero_bytes(s.xt, 16384);
    zero_bytes(s.h1t, 20480);
    zero_bytes(s.at, 32768);
    __syncthreads();
    for (int k = threadIdx.x; k < 128; k += blockDim.x) {
        put_bf16(s.xt, 48, k, 128, 1.0f);
        put_bf16(s.h1t, 64, k, 128, 1.0f);
        put_bf16(s.at, 64, k, 128, 1.0f);
    }
    if (threadIdx.x == 0) {
        tc::mbar_init(s.bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if ((threadIdx.x >> 5) == 0) {
        tc::tmem_alloc(s.slot, 512);
        tc::tmem_relinquish();
    }
    to_mma();
    const uint32_t tb = *s.slot;
    uint32_t phase = 0;
    const int r = threadIdx.x;
    const int nout = net.nout;
    float loss = 0.0f;
    bool first = true;
    const int64_t ntiles = (rows + kMlpTile - 1) / kMlpTile;
    for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int64_t r0 = t * kMlpTile;
        const bool valid = r0 + r < rows;
        // X and X^T (row r = sample; padded samples are zero and carry no loss)
        load_tile(s.x, feat + r0 * kMlpIn, kMlpTile, kMlpIn, rows - r0);
        __syncthreads();
        for (int q = threadIdx.x; q < kMlpTile * kMlpIn; q += blockDim.x) {
            const int smp = q / kMlpIn, f = q - smp * kMlpIn;
            const uint16_t v = *reinterpret_cast<const uint16_t*>(s.x + tc::core_offset(smp, f, kMlpIn));
            *reinterpret_cast<uint16_t*>(s.xt + tc::core_offset(f, smp, 128)) = v;
        }
        to_mma();
        if (r == 0) {
            issue_gemm(tb + kT1, s.x, s.w1, 64, kMlpIn, false);
            tc::mma_commit(s.bar);
        }
        if (!wait_all(s.bar, phase, err)) return abort_tc(s.bar, phase, tb, 512);
        const uint64_t m1 = epi_hidden(tb + kT1, s.bias, s.h);
        // H1^T for dW2
        for (int q = threadIdx.x; q < kMlpTile * kMlpHid; q += blockDim.x) {
            const int smp = q / kMlpHid, j = q - smp * kMlpHid;
            const uint16_t v = *reinterpret_cast<const uint16_t*>(s.h + tc::core_offset(smp, j, kMlpHid));
            *reinterpret_cast<uint16_t*>(s.h1t + tc::core_offset(j, smp, 128)) = v;
        }
        to_mma();
        if (r == 0) {
            issue_gemm(tb + kT2, s.h, s.w2, 64, kMlpHid, false);
            tc::mma_commit(s.bar);
        }
        if (!wait_all(s.bar, phase, err)) return abort_tc(s.bar, phase, tb, 512);
        const uint64_t m2 = epi_hidden(tb + kT2, s.bias + 64, s.h);
        __syncthreads();
        // H2^T for dW3^T (rows 0..63 of the shared transposed tile)
        for (int q = threadIdx.x; q < kMlpTile * kMlpHid; q += blockDim.x) {
            const int smp = q / kMlpHid, j = q - smp * kMlpHid;
            const uint16_t v = *reinterpret_cast<const uint16_t*>(s.h + tc::core_offset(smp, j, kMlpHid));
            *reinterpret_cast<uint16_t*>(s.at + tc::core_offset(j, smp, 128)) = v;
        }
        to_mma();
        if (r == 0) {
            issue_gemm(tb + kT1, s.h, s.w3, 16, kMlpHid, false);
            tc::mma_commit(s.bar);
        }
        if (!wait_all(s.bar, phase, err)) return abort_tc(s.bar, phase, tb, 512);
        // output layer: dY = (Y - T) on the used outputs of valid samples
        {
            float y[16], dy[16];
            tc::tmem_ld16(lane_base(tb + kT1), y);
#pragma unroll
            for (int v = 0; v < 16; ++v) {
                float d = 0.0f;
                if (valid && v < nout) d = (y[v] + s.bias[128 + v]) - target[(r0 + r) * kMlpOut + v];
                dy[v] = d;
                loss += d * d;
            }
            store8(s.dy, r, 0, 16, dy);
            store8(s.dy, r, 8, 16, dy + 8);
#pragma unroll
            for (int v = 0; v < 16; ++v) put_bf16(s.dyt, v, r, 128, dy[v]);
        }
        to_mma();
        if (r == 0) {
            issue_gemm(tb + kT2, s.dy, s.w3t, 64, 16, false);          // dH2 = dY W3
            issue_gemm(tb + kGW3, s.at, s.dyt, 16, 128, !first);       // dW3^T += H2^T dY
            tc::mma_commit(s.bar);
        }
        if (!wait_all(s.bar, phase, err)) return abort_tc(s.bar, phase, tb, 512);
        // dZ2 = dH2 * [Z2 > 0] -> s.h (A of dH1) and dZ2^T -> s.at (A of dW2)
#pragma unroll
        for (int c = 0; c < 64; c += 16) {
            float v[16];
            tc::tmem_ld16(lane_base(tb + kT2) + c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = ((m2 >> (c + i)) & 1u) ? v[i] : 0.0f;
            store8(s.h, r, c, 64, v);
            store8(s.h, r, c + 8, 64, v + 8);
#pragma unroll
            for (int i = 0; i < 16; ++i) put_bf16(s.at, c + i, r, 128, v[i]);
        }
        to_mma();
        if (r == 0) {
            issue_gemm(tb + kT1, s.h, s.w2t, 64, kMlpHid, false);      // dH1 = dZ2 W2
            issue_gemm(tb + kGW2, s.at, s.h1t, 80, 128, !first);      // dW2 += dZ2^T H1 (+ db2)
            tc::mma_commit(s.bar);
        }
        if (!wait_all(s.bar, phase, err)) return abort_tc(s.bar, phase, tb, 512);
        // dZ1 = dH1 * [Z1 > 0] -> s.at (A of dW1)
#pragma unroll
        for (int c = 0; c < 64; c += 16) {
            float v[16];
            tc::tmem_ld16(lane_base(tb + kT1) + c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) put_bf16(s.at, c + i, r, 128, ((m1 >> (c + i)) & 1u) ? v[i] : 0.0f);
        }
        to_mma();
        if (r == 0) {
            issue_gemm(tb + kGW1, s.at, s.xt, 64, 128, !first);       // dW1 += dZ1^T X (+ db1)
            tc::mma_commit(s.bar);
        }
        if (!wait_all(s.bar, phase, err)) return abort_tc(s.bar, phase, tb, 512);
        first = false;
        // the H2^T rows of s.at are rewritten by the next tile: restore nothing
        // (row 64 keeps its ones, rows 65.. stay zero)
    }
    // write this CTA's gradient partials (zero when it processed no tile)
    float* P = partials + int64_t(blockIdx.x) * (kMlpParams + 1);
    if (first) {
        for (int p = threadIdx.x; p < kMlpParams; p += blockDim.x) P[p] = 0.0f;
    } else {
        float v[16];
        // dW3^T: row r = input unit (r < 64), row 64 = db3
        tc::tmem_ld16(lane_base(tb + kGW3), v);
        if (r < 64) {
            for (int o = 0; o < kMlpOut; ++o) P[kOffW3 + o * kMlpHid + r] = v[o];
        } else if (r == 64) {
            for (int o = 0; o < kMlpOut; ++o) P[kOffB3 + o] = v[o];
        }
        // dW1: row r = output unit, columns 0..47 inputs, 48 bias
#pragma unroll
        for (int c = 0; c < 64; c += 16) {
            tc::tmem_ld16(lane_base(tb + kGW1) + c, v);
            if (r < 64)
                for (int i = 0; i < 16; ++i) {
                    const int col = c + i;
                    if (col < kMlpIn) P[kOffW1 + r * kMlpIn + col] = v[i];
                    else if (col == kMlpIn) P[kOffB1 + r] = v[i];
                }
        }
        // dW2: row r = output unit, columns 0..63 inputs, 64 bias
#pragma unroll
        for (int c = 0; c < 80; c += 16) {
            tc::tmem_ld16(lane_base(tb + kGW2) + c, v);
            if (r < 64)
                for (int i = 0; i < 16; ++i) {
                    const int col = c + i;
                    if (col < kMlpHid) P[kOffW2 + r * kMlpHid + col] = v[i];
                    else if (col == kMlpHid) P[kOffB2 + r] = v[i];
                }
        }
    }
    // loss partial (fixed-order block sum)
    s.red[r] = loss;
    __syncthreads();
    if (r == 0) {
        float acc = 0.0f;
        for (int i = 0; i < 128; ++i) acc += s.red[i];
        P[kMlpParams] = acc;
    }
    tc::fence_before_sync();
    __syncthreads();
    if ((threadIdx.x >> 5) == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tb, 512);
    }
}

__global__ void k_mlp_adam(float* params, float* m, float* v, const float* __restrict__ partials, int nparts,
                           double inv_count, float lr, float b1, float b2, float eps, float c1, float c2, bool adam,
                           float* grad_out, float* loss_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > kMlpParams) return;
    double acc = 0.0;
    for (int c = 0; c < nparts; ++c) acc += double(partials[int64_t(c) * (kMlpParams + 1) + p]);
    if (p == kMlpParams) {
        if (loss_out) *loss_out = float(acc * inv_count);
        return;
    }
    const float g = float(2.0 * acc * inv_count);  // d/dtheta of mean (y - t)^2
    if (grad_out) grad_out[p] = g;
    if (!adam) return;
    const float mi = b1 * m[p] + (1.0f - b1) * g;
    const float vi = b2 * v[p] + (1.0f - b2) * g * g;
    m[p] = mi;
    v[p] = vi;
    params[p] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_mlp_sync_bf16(const float* __restrict__ params, uint16_t* w1, uint16_t* w2, uint16_t* w3) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kMlpHid * kMlpIn) w1[i] = f2bf(params[kOffW1 + i]);
    if (i < kMlpHid * kMlpHid) w2[i] = f2bf(params[kOffW2 + i]);
    if (i < kMlpOut * kMlpHid) w3[i] = f2bf(params[kOffW3 + i]);
}

}  // namespace

void launch_tc_selftest(const uint16_t* A, const uint16_t* B, float* D, int N, int K, int* err, cudaStream_t s) {
    const int bytes = 128 * K * 2 + 64 * K * 2 + 16;
    cudaFuncSetAttribute(k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    k_tc_selftest<<<1, 128, bytes, s>>>(A, B, D, N, K, err);
}

void launch_mlp_forward(const MlpDev& net, const uint16_t* feat, int64_t rows, const double* scale, int nv,
                        double* out, int* err, int grid, cudaStream_t s) {
    if (rows <= 0) return;
    cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem);
    const int64_t ntiles = (rows + kMlpTile - 1) / kMlpTile;
    const int g = static_cast<int>(std::min<int64_t>(ntiles, grid));
    k_mlp_forward<<<g, 128, kFwdSmem, s>>>(net, feat, rows, scale, nv, out, err);
}

void launch_mlp_grad(const MlpDev& net, const uint16_t* feat, const float* target, int64_t rows, float* partials,
                     int* err, int grid, cudaStream_t s) {
    cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem);
    k_mlp_grad<<<grid, 128, kTrainSmem, s>>>(net, feat, target, rows, partials, err);
}

void launch_mlp_adam(float* params, float* m, float* v, uint16_t* w1, uint16_t* w2, uint16_t* w3,
                     const float* partials, int nparts, double inv_count, float lr, float beta1, float beta2,
                     float eps, int step, bool adam, float* grad_out, float* loss_out, cudaStream_t s) {
    const float c1 = 1.0f - powf(beta1, float(step)), c2 = 1.0f - powf(beta2, float(step));
    k_mlp_adam<<<(kMlpParams + 1 + 255) / 256, 256, 0, s>>>(params, m, v, partials, nparts, inv_count, lr, beta1,
                                                             beta2, eps, c1, c2, adam, grad_out, loss_out);
    if (adam) launch_mlp_sync_bf16(params, w1, w2, w3, s);
}

void launch_mlp_sync_bf16(const float* params, uint16_t* w1, uint16_t* w2, uint16_t* w3, cudaStream_t s) {
    k_mlp_sync_bf16<<<(kMlpHid * kMlpHid + 255) / 256, 256, 0, s>>>(params, w1, w2, w3);
}

}  // namespace cfdg
