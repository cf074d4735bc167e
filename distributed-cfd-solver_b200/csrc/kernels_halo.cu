// Halo message packing: the SoA cell fields of the listed cells into one
// AoS message (cell-major, nvars values a cell) and back, the device form of
// pack_soa_to_aos / unpack_aos_to_soa (src/fields/halo.cpp:26-124).  One
// thread per (cell, variable) entry of the message, so consecutive threads
// write (pack) or read (unpack) consecutive message entries.
#include "halo.hpp"

namespace cfdg {

namespace {

__global__ void k_halo_pack(int32_t n, const int32_t* __restrict__ idx, HaloFields f, int nvars,
                            double* __restrict__ msg) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(n) * nvars) return;
    const int32_t i = static_cast<int32_t>(t / nvars);
    const int v = static_cast<int>(t - int64_t(i) * nvars);
    msg[t] = f.p[v][__ldg(idx + i)];
}

__global__ void k_halo_unpack(int32_t n, const int32_t* __restrict__ idx, const double* __restrict__ msg, int nvars,
                              HaloFields f) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(n) * nvars) return;
    const int32_t i = static_cast<int32_t>(t / nvars);
    const int v = static_cast<int>(t - int64_t(i) * nvars);
    f.p[v][__ldg(idx + i)] = msg[t];
}

// Block vectors (x[row * bs + v], the Krylov vectors' layout): the listed
// rows' blocks back to back, as the reference's vector layout packs them
// (include/cfd/linalg/vector_layout.hpp:170-250).
__global__ void k_halo_pack_blocks(int32_t n, const int32_t* __restrict__ idx, const double* __restrict__ x, int bs,
                                   double* __restrict__ msg) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(n) * bs) return;
    const int32_t i = static_cast<int32_t>(t / bs);
    const int v = static_cast<int>(t - int64_t(i) * bs);
    msg[t] = x[int64_t(__ldg(idx + i)) * bs + v];
}

__global__ void k_halo_unpack_blocks(int32_t n, const int32_t* __restrict__ idx, const double* __restrict__ msg, int bs,
                                     double* __restrict__ x) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(n) * bs) return;
    const int32_t i = static_cast<int32_t>(t / bs);
    const int v = static_cast<int>(t - int64_t(i) * bs);
    x[int64_t(__ldg(idx + i)) * bs + v] = msg[t];
}

}  // namespace

void launch_halo_pack_blocks(int32_t n, const int32_t* idx, const double* x, int bs, double* msg, cudaStream_t s) {
    const int64_t len = int64_t(n) * bs;
    if (len > 0) k_halo_pack_blocks<<<grid_for(len, 256), 256, 0, s>>>(n, idx, x, bs, msg);
}

void launch_halo_unpack_blocks(int32_t n, const int32_t* idx, const double* msg, int bs, double* x, cudaStream_t s) {
    const int64_t len = int64_t(n) * bs;
    if (len > 0) k_halo_unpack_blocks<<<grid_for(len, 256), 256, 0, s>>>(n, idx, msg, bs, x);
}

void launch_halo_pack(int32_t n, const int32_t* idx, const HaloFields& f, int nvars, double* msg, cudaStream_t s) {
    const int64_t len = int64_t(n) * nvars;
    if (len > 0) k_halo_pack<<<grid_for(len, 256), 256, 0, s>>>(n, idx, f, nvars, msg);
}

void launch_halo_unpack(int32_t n, const int32_t* idx, const double* msg, int nvars, const HaloFields& f,
                        cudaStream_t s) {
    const int64_t len = int64_t(n) * nvars;
    if (len > 0) k_halo_unpack<<<grid_for(len, 256), 256, 0, s>>>(n, idx, msg, nvars, f);
}

}  // namespace cfdg
