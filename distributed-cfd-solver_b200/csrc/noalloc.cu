// Allocation-free residual norms: cfdg_residual_norms_noalloc.
//
// For callers that cannot allocate device memory themselves or through the
// library: a host code that hands the whole device memory budget to its
// own pool allocator and forbids any other cudaMalloc, or a monitoring hook
// called between the solver's kernels where a cudaMalloc/cudaFree would
// synchronise the device and stall the pipeline.  They pass the residual
// array they already own and get the per-variable L2 norms back; the
// per-block partial sums live in a static device array of this file.
//
// Limits: nvars <= 6 and n_cells <= 4,194,304 (one partial per 256 cells,
// 16,384 blocks x 6 variables = 768 KiB of scratch, held by every GPU that
// loads the library until the process exits).  Every call shares the
// array; a call writes every partial it reads before reading it, so nothing
// has to start at zero, but calls that overlap on the GPU (two streams, two
// host threads) race on it.  The first call on a device looks up the
// array's device address on that device; make that first call outside any
// stream capture.  The address is cached for the process's lifetime, so a
// cudaDeviceReset (which re-creates the primary context and reloads this
// module) leaves it stale: do not call the entry point after one.
#include <cuda_runtime.h>

#include <mutex>

#include "cfdg.h"
#include "kernels.hpp"
#include "solver.hpp"

namespace cfdg {
namespace {

constexpr int kNoAllocBlock = 256;
constexpr int kNoAllocMaxBlocks = 16384;
constexpr int kNoAllocMaxVars = 6;
constexpr int64_t kNoAllocMaxCells = int64_t(kNoAllocMaxBlocks) * kNoAllocBlock;  // 4,194,304
constexpr int kNoAllocSlots = kNoAllocMaxBlocks * kNoAllocMaxVars + 8;              // + 8 result slots

// Scratch: block partials [block][var], then the nvars results.  In host
// code this name is a host-side stand-in; kernels get the device address.
__device__ __align__(256) double g_noalloc_scratch[kNoAllocSlots];

constexpr int kMaxDevices = 64;
double* g_scratch_dev[kMaxDevices] = {};
std::mutex g_scratch_mutex;

template <int NV>
__global__ void __launch_bounds__(kNoAllocBlock) k_norm_partials_noalloc(int32_t n, const double* __restrict__ res,
                                                                        double* __restrict__ scratch) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    double sq[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const double r = (c < n) ? res[int64_t(v) * n + c] : 0.0;
        sq[v] = r * r;
    }
    block_reduce_store<NV, kNoAllocBlock>(sq, scratch + size_t(blockIdx.x) * NV);
}

// Warp v sums column v of the partials in a fixed order.
__global__ void k_norm_finalize_noalloc(int nblocks, int nv, double scale, double* __restrict__ scratch) {
    const int v = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (v >= nv) return;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += scratch[size_t(b) * nv + v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) scratch[size_t(kNoAllocMaxBlocks) * kNoAllocMaxVars + v] = sqrt(s * scale);
}

// Device address of the scratch on the current device, looked up once.
int scratch_for_current_device(double** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CFDG_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_dev[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return CFDG_ERR_CUDA;
        g_scratch_dev[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_dev[dev];
    return CFDG_OK;
}

}  // namespace
}  // namespace cfdg

extern "C" int cfdg_residual_norms_noalloc(const double* res_d, int32_t n_cells, int32_t nvars, void* stream,
                                           double* l2_h) {
    using namespace cfdg;
    if (!res_d || !l2_h || n_cells <= 0 || nvars < 1) {
        set_error("cfdg_residual_norms_noalloc: null pointer or empty size");
        return CFDG_ERR_INVALID;
    }
    if (nvars > kNoAllocMaxVars || int64_t(n_cells) > kNoAllocMaxCells) {
        set_error("cfdg_residual_norms_noalloc: nvars must be <= 6 and n_cells <= 4194304 (static scratch limit)");
        return CFDG_ERR_INVALID;
    }
    double* scratch = nullptr;
    if (scratch_for_current_device(&scratch) != CFDG_OK) {
        cudaGetLastError();
        set_error("cfdg_residual_norms_noalloc: device address of the static scratch unavailable");
        return CFDG_ERR_CUDA;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nblocks = static_cast<int>((int64_t(n_cells) + kNoAllocBlock - 1) / kNoAllocBlock);
    switch (nvars) {
        case 1: k_norm_partials_noalloc<1><<<nblocks, kNoAllocBlock, 0, s>>>(n_cells, res_d, scratch); break;
        case 2: k_norm_partials_noalloc<2><<<nblocks, kNoAllocBlock, 0, s>>>(n_cells, res_d, scratch); break;
        case 3: k_norm_partials_noalloc<3><<<nblocks, kNoAllocBlock, 0, s>>>(n_cells, res_d, scratch); break;
        case 4: k_norm_partials_noalloc<4><<<nblocks, kNoAllocBlock, 0, s>>>(n_cells, res_d, scratch); break;
        case 5: k_norm_partials_noalloc<5><<<nblocks, kNoAllocBlock, 0, s>>>(n_cells, res_d, scratch); break;
        default: k_norm_partials_noalloc<6><<<nblocks, kNoAllocBlock, 0, s>>>(n_cells, res_d, scratch); break;
    }
    k_norm_finalize_noalloc<<<1, 32 * kNoAllocMaxVars, 0, s>>>(nblocks, nvars, 1.0 / double(n_cells), scratch);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(l2_h, scratch + size_t(kNoAllocMaxBlocks) * kNoAllocMaxVars, sizeof(double) * nvars,
                            cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error(std::string("cfdg_residual_norms_noalloc: ") + cudaGetErrorString(e));
        return CFDG_ERR_CUDA;
    }
    return CFDG_OK;
}
