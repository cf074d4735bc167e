// Block-sparse linear algebra on the device: BSR SpMV with fused inner
// products, block LU of the diagonal, SGS sweeps over row lists (levels or
// colours), and the BiCGSTAB vector kernels with device-side scalar logic.
//
// References (maksim-movsisyan/Distributed-cfd-solver):
//   bsr_spmv<BS>          include/cfd/linalg/bsr_helpers.hpp:138-203
//   lu_factor_block       include/cfd/linalg/bsr_helpers.hpp:278-321
//   lu_solve_block<BS>    include/cfd/linalg/bsr_helpers.hpp:324-353
//   bsr_sgs_sweep<BS>     include/cfd/linalg/bsr_helpers.hpp:389-435
//   BiCGSTAB::solve       src/linalg/bicgstab.cpp:42-201
#include <algorithm>
#include <atomic>

#include <cooperative_groups.h>

#include "kernels.hpp"
#include "krylov.hpp"

namespace cfdg {

namespace {

template <typename MT>
__device__ __forceinline__ double ld(const MT* p) { return static_cast<double>(__ldg(p)); }

// Row ii of a BS x BS block (BS consecutive values) into registers.  Rows of
// 6x6 blocks start on 48-byte (FP64) / 24-byte (FP32) boundaries and load as
// pairs.
template <typename MT, int BS>
__device__ __forceinline__ void load_block_row(const MT* __restrict__ a, double (&out)[BS]) {
    if constexpr (BS == 6 && sizeof(MT) == 8) {
        const double2* p = reinterpret_cast<const double2*>(a);
#pragma unroll
        for (int h = 0; h < 3; ++h) {
            const double2 v = __ldg(p + h);
            out[2 * h] = v.x;
            out[2 * h + 1] = v.y;
        }
    } else if constexpr (BS == 6 && sizeof(MT) == 4) {
        const float2* p = reinterpret_cast<const float2*>(a);
#pragma unroll
        for (int h = 0; h < 3; ++h) {
            const float2 v = __ldg(p + h);
            out[2 * h] = v.x;
            out[2 * h + 1] = v.y;
        }
    } else {
#pragma unroll
        for (int j = 0; j < BS; ++j) out[j] = ld(a + j);
    }
}

// One block's entries of a vector (BS consecutive doubles) through the
// read-only path: the neighbour entries a sweep or product reads are not
// written during the launch (rows of one colour or level are never
// neighbours).  6-entry blocks are 16-byte aligned and load as pairs.
// COHERENT: through L2 only (ld.global.cg), for entries other SMs wrote
// earlier in the same launch (the cooperative level sweep).
template <int BS, bool COHERENT = false>
__device__ __forceinline__ void load_vec(const double* __restrict__ x, double (&out)[BS]) {
    if constexpr (BS == 6 || BS == 4) {
        const double2* p = reinterpret_cast<const double2*>(x);
#pragma unroll
        for (int h = 0; h < BS / 2; ++h) {
            const double2 v = COHERENT ? __ldcg(p + h) : __ldg(p + h);
            out[2 * h] = v.x;
            out[2 * h + 1] = v.y;
        }
    } else {
#pragma unroll
        for (int j = 0; j < BS; ++j) out[j] = COHERENT ? __ldcg(x + j) : __ldg(x + j);
    }
}

// acc (+|-)= sum over blocks k in [k0, k1) of A_k[ii][:] . x_col(k) in
// ascending block order, each block's partial sum formed first (the
// arithmetic of the sequential sweep and product).  The block row and the
// neighbour's x block load as 16-byte pairs for 6x6 blocks (measured on the
// SA plate: SGS 0.73 -> 0.80 of the copy bandwidth); other block sizes keep
// scalar loads, which measured faster for 5x5 (FP32 tet bump).
template <typename MT, int BS, bool SUB, bool COHERENT = false>
__device__ __forceinline__ double block_row_dot(const BsrView& A, const MT* __restrict__ vals, const double* x,
                                                int ii, int32_t k0, int32_t k1, double acc) {
    for (int32_t k = k0; k < k1; ++k) {
        double t = 0.0;
        if constexpr (BS == 6) {
            double a[BS], xb[BS];
            load_block_row<MT, BS>(vals + int64_t(k) * (BS * BS) + ii * BS, a);
            load_vec<BS, COHERENT>(x + int64_t(__ldg(A.cols + k)) * BS, xb);
#pragma unroll
            for (int jj = 0; jj < BS; ++jj) t += a[jj] * xb[jj];
        } else {
            const MT* a = vals + int64_t(k) * (BS * BS) + ii * BS;
            const double* xb = x + int64_t(A.cols[k]) * BS;
#pragma unroll
            for (int jj = 0; jj < BS; ++jj) t += ld(a + jj) * (COHERENT ? __ldcg(xb + jj) : xb[jj]);
        }
        acc = SUB ? acc - t : acc + t;
    }
    return acc;
}

// --------------------------------------------------------------- SpMV
// Vector kernels and the SpMV run a fixed grid of at most kVecGridCap
// blocks (8 resident 256-thread blocks on each of 148 SMs) striding over
// the vector, so that the per-block partial sums of the fused inner
// products number at most kVecGridCap and the single-block finalisers read
// them in a few loads per thread.  The grid depends only on the length, so
// the summation order, and the result, is the same run to run.
constexpr int kVecThreads = 256;
constexpr int64_t kVecGridCap = 148 * 8;

inline unsigned vec_grid(int64_t len) {
    const int64_t g = grid_for(len, kVecThreads);
    return static_cast<unsigned>(g < kVecGridCap ? g : kVecGridCap);
}

// One thread per (block row, component): y_i[ii] = alpha * sum_k sum_jj
// A_k[ii][jj] x_col(k)[jj] + beta * y.  Optional fused dot products of y
// (or other vectors) for the Krylov scalars, reduced per block.
// Rows [row_begin, n) (row_begin > 0: the rows left after the fused
// product of the last SGS pass).
template <typename MT, int BS, int ND>
__global__ void __launch_bounds__(kVecThreads) k_spmv(BsrView A, const MT* __restrict__ vals,
                                                      const double* __restrict__ x, double* __restrict__ y,
                                                      double alpha, double beta, DotSpec ds,
                                                      double* __restrict__ partials, const int* __restrict__ active,
                                                      int32_t row_begin) {
    if (active && *active != 0) return;
    const int64_t N = int64_t(A.n) * BS;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    double pr[ND > 0 ? ND : 1];
#pragma unroll
    for (int k = 0; k < (ND > 0 ? ND : 1); ++k) pr[k] = 0.0;
    for (int64_t t = int64_t(row_begin) * BS + int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < N; t += stride) {
        const int32_t row = static_cast<int32_t>(t / BS);
        const int ii = static_cast<int>(t % BS);
        double acc = 0.0;
        const int32_t k1 = A.row_ptr[row + 1];
        for (int32_t k = A.row_ptr[row]; k < k1; ++k) {
            const MT* a = vals + int64_t(k) * (BS * BS) + ii * BS;
            const double* xb = x + int64_t(A.cols[k]) * BS;
            double s = 0.0;
#pragma unroll
            for (int jj = 0; jj < BS; ++jj) s += ld(a + jj) * xb[jj];
            acc += s;
        }
        double yv;
        if (alpha == 1.0 && beta == 0.0) yv = acc;
        else if (beta == 1.0) yv = y[t] + alpha * acc;
        else if (beta == 0.0) yv = alpha * acc;
        else yv = alpha * acc + beta * y[t];
        y[t] = yv;
        if constexpr (ND > 0) {
#pragma unroll
            for (int k = 0; k < ND; ++k) {
                const double a = ds.a[k] ? ds.a[k][t] : yv;
                const double b = ds.b[k] ? ds.b[k][t] : yv;
                pr[k] += a * b;
            }
        }
    }
    if constexpr (ND > 0) block_reduce_store<ND, kVecThreads>(pr, partials + size_t(blockIdx.x) * ND);
}

// -------------------------------------------------------- block LU setup
// One thread per block row; the CTA's 128 diagonal blocks are staged through
// shared memory so that the loads (one block per 25 / 36 consecutive
// threads) and the stores (the CTA's LU blocks are one contiguous range) are
// coalesced.
constexpr int kLuThreads = 128;

// INV: the factors are used once more to form the explicit inverse D^-1
// (A x = e_c column by column), which is stored instead of the factors; the
// multicolour sweep then applies D^-1 as a block-row product.
// Occupancy bound per block size: the 6x6 factor, pivots and inverse
// column of a thread spill below ~170 registers, the 5x5 ones below ~128.
template <typename MT, int BS, bool INV>
__global__ void __launch_bounds__(kLuThreads, BS == 6 ? 3 : 4) k_lu(BsrView A, const MT* __restrict__ vals, MT* __restrict__ lu,
                                                   int8_t* __restrict__ piv, int* __restrict__ err) {
    constexpr int B2 = BS * BS;
    constexpr int SP = B2 % 2 == 0 ? B2 + 1 : B2;  // odd row stride: thread-per-row accesses hit distinct banks
    __shared__ MT sm[kLuThreads * SP];
    const int32_t r0 = blockIdx.x * kLuThreads;
    const int32_t nrows = min(kLuThreads, A.n - r0);
    for (int q = threadIdx.x; q < nrows * B2; q += kLuThreads) {
        const int row = q / B2, e = q - row * B2;
        sm[row * SP + e] = vals[int64_t(A.diag[r0 + row]) * B2 + e];
    }
    __syncthreads();
    const int32_t i = r0 + threadIdx.x;
    const bool act = threadIdx.x < nrows;
    double a[BS * BS];
    if (act) {
#pragma unroll
        for (int e = 0; e < BS * BS; ++e) a[e] = static_cast<double>(sm[threadIdx.x * SP + e]);
    } else {
#pragma unroll
        for (int e = 0; e < BS * BS; ++e) a[e] = (e % (BS + 1) == 0) ? 1.0 : 0.0;
    }
    int8_t pv[BS];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < BS; ++k) {
        int m = k;
        double mx = fabs(a[k * BS + k]);
#pragma unroll
        for (int r = k + 1; r < BS; ++r) {
            const double v = fabs(a[r * BS + k]);
            if (v > mx) {
                mx = v;
                m = r;
            }
        }
        pv[k] = static_cast<int8_t>(m);
        if (mx == 0.0) ok = false;
        // row swap by selects (no data-dependent branch, so a[] stays in
        // registers)
#pragma unroll
        for (int r = k + 1; r < BS; ++r) {
            const bool sw = (r == m);
#pragma unroll
            for (int j = 0; j < BS; ++j) {
                const double ak = a[k * BS + j], ar = a[r * BS + j];
                a[k * BS + j] = sw ? ar : ak;
                a[r * BS + j] = sw ? ak : ar;
            }
        }
        const double inv_d = 1.0 / a[k * BS + k];
#pragma unroll
        for (int r = k + 1; r < BS; ++r) {
            const double l = a[r * BS + k] * inv_d;
            a[r * BS + k] = l;
#pragma unroll
            for (int j = k + 1; j < BS; ++j) a[r * BS + j] -= l * a[k * BS + j];
        }
    }
    __syncthreads();  // every thread has read its block
    if (act) {
        if constexpr (INV) {
            // the U diagonal's reciprocals once: BS divisions instead of BS*BS
            double rd[BS];
#pragma unroll
            for (int r = 0; r < BS; ++r) rd[r] = 1.0 / a[r * BS + r];
#pragma unroll
            for (int c = 0; c < BS; ++c) {
                double x[BS];
#pragma unroll
                for (int j = 0; j < BS; ++j) x[j] = (j == c) ? 1.0 : 0.0;
#pragma unroll
                for (int k = 0; k < BS; ++k) {
#pragma unroll
                    for (int j = k + 1; j < BS; ++j) {
                        const bool sw = (j == pv[k]);
                        const double xk = x[k], xj = x[j];
                        x[k] = sw ? xj : xk;
                        x[j] = sw ? xk : xj;
                    }
                }
#pragma unroll
                for (int r = 1; r < BS; ++r)
#pragma unroll
                    for (int j = 0; j < r; ++j) x[r] -= a[r * BS + j] * x[j];
#pragma unroll
                for (int r = BS - 1; r >= 0; --r) {
#pragma unroll
                    for (int j = r + 1; j < BS; ++j) x[r] -= a[r * BS + j] * x[j];
                    x[r] = x[r] * rd[r];
                }
#pragma unroll
                for (int r = 0; r < BS; ++r) sm[threadIdx.x * SP + r * BS + c] = static_cast<MT>(x[r]);
            }
        } else {
#pragma unroll
            for (int e = 0; e < BS * BS; ++e) sm[threadIdx.x * SP + e] = static_cast<MT>(a[e]);
        }
#pragma unroll
        for (int k = 0; k < BS; ++k) piv[int64_t(i) * BS + k] = pv[k];
        // +(i+1): zero pivot (singular block); -(i+1): non-finite entries
        bool finite = true;
#pragma unroll
        for (int e = 0; e < BS * BS; ++e) finite = finite && isfinite(a[e]);
        if (!ok) {
            atomicCAS(err, 0, i + 1);
        } else if (!finite) {
            atomicCAS(err, 0, -(i + 1));
        }
    }
    __syncthreads();
    MT* dst = lu + int64_t(r0) * B2;
    for (int q = threadIdx.x; q < nrows * B2; q += kLuThreads) {
        const int row = q / B2, e = q - row * B2;
        dst[q] = sm[row * SP + e];
    }
}

// Pivoted forward/backward substitution of one block (lu_solve_block) in
// registers; b holds the right-hand side on entry and the solution on exit.
template <typename MT, int BS, bool SMEM = false>
__device__ __forceinline__ void lu_solve(const MT* __restrict__ lu, const int8_t* __restrict__ piv, double (&b)[BS]) {
    auto L = [&](int idx) -> double { return SMEM ? static_cast<double>(lu[idx]) : ld(lu + idx); };
#pragma unroll
    for (int k = 0; k < BS; ++k) {
        const int p = piv[k];
        double bp = b[k];
#pragma unroll
        for (int j = k + 1; j < BS; ++j)
            if (j == p) bp = b[j];
        const double bk = b[k];
        b[k] = bp;
#pragma unroll
        for (int j = k + 1; j < BS; ++j)
            if (j == p) b[j] = bk;
    }
#pragma unroll
    for (int i = 1; i < BS; ++i) {
        double s = b[i];
#pragma unroll
        for (int j = 0; j < i; ++j) s -= L(i * BS + j) * b[j];
        b[i] = s;
    }
#pragma unroll
    for (int i = BS - 1; i >= 0; --i) {
        double s = b[i];
#pragma unroll
        for (int j = i + 1; j < BS; ++j) s -= L(i * BS + j) * b[j];
        b[i] = s / L(i * BS + i);
    }
}

// One SGS pass over a row list.  A group of BS lanes owns one row: lane ii
// accumulates component ii of s = r_i - sum_{k != diag} A_ik z_k (columns in
// ascending order, as the sequential sweep), the group exchanges s by warp
// shuffles, and each lane solves the pivoted LU system and keeps its entry.
// MODE 1 skips the neighbour sum (all neighbour z are still zero).
// INV: `lu` holds the explicit inverse D^-1 (multicolour ordering), applied
// as a block-row product: five loads per lane instead of the whole factor.
// MODE 2 and 3 are the two halves of the first symmetric sweep of a
// colour-ordered matrix (every colour a contiguous row range, colours
// ascending, so "column < row" means "earlier colour"):
//   MODE 2 (forward)  y_i = D_i^-1 (r_i - sum_{k < diag} A_ik y_k);
//   MODE 3 (backward) z_i = y_i - D_i^-1 sum_{k > diag} A_ik z_k,
// which equals the full-row backward update D_i^-1 (r_i - sum_lower A y -
// sum_upper A z) because (D + L) y = r, and reads neither r nor the lower
// blocks.
template <typename MT, int BS, int MODE, bool INV>
__global__ void __launch_bounds__(256, (INV && BS <= 5) ? 8 : 6) k_sgs_rows(BsrView A, const MT* __restrict__ vals, const MT* __restrict__ lu,
                                                  const int8_t* __restrict__ piv, const int32_t* __restrict__ rows,
                                                  int32_t row0, int32_t n_rows, const double* __restrict__ r,
                                                  double* __restrict__ z, const int* __restrict__ active) {
    if (active && *active != 0) return;
    constexpr int GPW = 32 / BS;
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int grp = lane / BS, ii = lane - grp * BS;
    const int64_t slot = warp * GPW + grp;
    const bool act = (grp < GPW) && (slot < n_rows);
    int32_t i = 0;
    double s = 0.0;
    if (act) {
        i = rows ? rows[slot] : row0 + static_cast<int32_t>(slot);  // null: a contiguous group
        s = (MODE == 3) ? 0.0 : r[int64_t(i) * BS + ii];
        if (MODE != 1) {
            const int32_t d = A.diag[i];
            if (MODE == 0) {  // lower then upper blocks, skipping the diagonal
                s = block_row_dot<MT, BS, true>(A, vals, z, ii, A.row_ptr[i], d, s);
                s = block_row_dot<MT, BS, true>(A, vals, z, ii, d + 1, A.row_ptr[i + 1], s);
            } else {
                const int32_t k0 = (MODE == 3) ? d + 1 : A.row_ptr[i];
                const int32_t k1 = (MODE == 2) ? d : A.row_ptr[i + 1];
                s = block_row_dot<MT, BS, true>(A, vals, z, ii, k0, k1, s);
            }
        }
    }
    double b[BS];
    const int base = (grp < GPW ? grp : 0) * BS;
#pragma unroll
    for (int j = 0; j < BS; ++j) b[j] = __shfl_sync(0xffffffffu, s, base + j);
    if (act) {
        double out;
        if constexpr (INV) {  // row ii of D^-1 times s
            const MT* di = lu + int64_t(i) * (BS * BS) + ii * BS;
            out = 0.0;
#pragma unroll
            for (int j = 0; j < BS; ++j) out += ld(di + j) * b[j];
        } else {
            lu_solve<MT, BS>(lu + int64_t(i) * (BS * BS), piv + int64_t(i) * BS, b);
            out = b[0];
#pragma unroll
            for (int j = 1; j < BS; ++j)
                if (j == ii) out = b[j];
        }
        // MODE 3: b solved D x = -sum_upper A z, so z_i = y_i + x
        if (MODE == 3) out = z[int64_t(i) * BS + ii] + out;
        z[int64_t(i) * BS + ii] = out;
    }
}

// The level-scheduled sweep (the reference's sequential order) in one
// cooperative launch: the resident grid walks the forward levels, then the
// backward levels, with a grid-wide barrier between levels instead of a
// kernel boundary.  A level's rows are independent but few (~1-7 thousand),
// so the time per level is the latency of one row's dependent loads; one
// warp takes a row and its lanes form KS = 32/BS groups of BS lanes, group
// g computing the block products t_k = A_k[ii][:] . z_col(k) of blocks
// k0+g, k0+g+KS, ... in parallel (one round trip for all of a row's blocks
// instead of one per block).  Group 0 then subtracts them from r in
// ascending block order by shuffles, which is the arithmetic of k_sgs_rows
// MODE 0 (and of the sequential sweep) to the bit, and solves the pivoted
// LU system.  z entries written in one level are read by later levels on
// other SMs, so z is read through L2 (ld.global.cg), never from a stale L1
// line.  Every loop is bounded by the level, row and block counts, and the
// cooperative launch makes every block resident, so every barrier is
// reached by all blocks.
// `fwd_rows` / `bwd_rows` are the passes' rows in level order as int4
// records (row, first block, end of the row's blocks, diagonal block), so a
// row's structure is one 16-byte load rather than a row-list load followed
// by the row-pointer and diagonal loads.
template <typename MT, int BS>
__global__ void __launch_bounds__(256) k_sgs_level_coop(BsrView A, const MT* __restrict__ vals,
                                                        const MT* __restrict__ lu, const int8_t* __restrict__ piv,
                                                        const int4* __restrict__ fwd_rows,
                                                        const int32_t* __restrict__ fwd_off, int n_fwd,
                                                        const int4* __restrict__ bwd_rows,
                                                        const int32_t* __restrict__ bwd_off, int n_bwd,
                                                        const double* __restrict__ r, double* z,
                                                        const int* __restrict__ active) {
    if (active && *active != 0) return;  // the same value for every block: all return before the first barrier
    namespace cg = cooperative_groups;
    cg::grid_group grid = cg::this_grid();
    constexpr int KS = 32 / BS;  // block products in flight per row
    const int lane = threadIdx.x & 31;
    const int64_t warp = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    const int grp = lane / BS, ii = lane - grp * BS;
    const bool in_grp = grp < KS;
    for (int pass = 0; pass < 2; ++pass) {
        const int4* rows = pass ? bwd_rows : fwd_rows;
        const int32_t* off = pass ? bwd_off : fwd_off;
        const int ng = pass ? n_bwd : n_fwd;
        for (int g = 0; g < ng; ++g) {
            const int32_t o0 = off[g];
            const int64_t nr = off[g + 1] - o0;
            for (int64_t slot = warp; slot < nr; slot += nwarps) {  // one row per warp: warp-uniform
                const int4 rec = __ldg(rows + o0 + slot);
                const int32_t i = rec.x, k0 = rec.y, k1 = rec.z, d = rec.w;
                double s = (grp == 0) ? r[int64_t(i) * BS + ii] : 0.0;
                for (int32_t kc = k0; kc < k1; kc += KS) {  // chunks of KS blocks, warp-uniform
                    const int32_t k = kc + grp;
                    double t = 0.0;
                    if (in_grp && k < k1 && k != d) {
                        double a[BS], xb[BS];
                        load_block_row<MT, BS>(vals + int64_t(k) * (BS * BS) + ii * BS, a);
                        load_vec<BS, true>(z + int64_t(__ldg(A.cols + k)) * BS, xb);
#pragma unroll
                        for (int jj = 0; jj < BS; ++jj) t += a[jj] * xb[jj];
                    }
                    // ascending block order: group q holds block kc + q
#pragma unroll
                    for (int q = 0; q < KS; ++q) {
                        const double tq = __shfl_sync(0xffffffffu, t, q * BS + (ii < BS ? ii : 0));
                        if (kc + q < k1 && kc + q != d) s -= tq;
                    }
                }
                double b[BS];
#pragma unroll
                for (int j = 0; j < BS; ++j) b[j] = __shfl_sync(0xffffffffu, s, j);
                if (grp == 0) {
                    lu_solve<MT, BS>(lu + int64_t(i) * (BS * BS), piv + int64_t(i) * BS, b);
                    double out = b[0];
#pragma unroll
                    for (int j = 1; j < BS; ++j)
                        if (j == ii) out = b[j];
                    z[int64_t(i) * BS + ii] = out;
                }
            }
            grid.sync();
        }
    }
}

// The last backward pass of a split multicolour sweep (colour 0, rows
// [0, n_rows), every neighbour of a later colour and already final) fused
// with the product y = A z on those rows.  The pass computes
// t = sum_{k > diag} A_ik z_k and z_i = y_i - D_i^-1 t (MODE 3 with D^-1);
// all of row i's off-diagonal blocks are then in t, so
// (A z)_i = t + A_ii z_i costs one more block instead of the row's blocks
// again.  Dot products of the result as k_spmv; the grid strides over the
// rows so the partials number at most kVecGridCap.
template <typename MT, int BS, int ND>
__global__ void __launch_bounds__(256, BS <= 5 ? 6 : 5) k_sgs_last_spmv(BsrView A, const MT* __restrict__ vals,
                                                                       const MT* __restrict__ dinv, int32_t n_rows,
                                                                       double* __restrict__ z, double* __restrict__ y,
                                                                       DotSpec ds, double* __restrict__ partials,
                                                                       const int* __restrict__ active) {
    if (active && *active != 0) return;
    constexpr int GPW = 32 / BS;
    const int lane = threadIdx.x & 31;
    const int grp = lane / BS, ii = lane - grp * BS;
    const int base = (grp < GPW ? grp : 0) * BS;
    const int64_t warps = (int64_t(gridDim.x) * blockDim.x) >> 5;
    double pr[ND > 0 ? ND : 1];
#pragma unroll
    for (int k = 0; k < (ND > 0 ? ND : 1); ++k) pr[k] = 0.0;
    for (int64_t w = (int64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; w * GPW < n_rows; w += warps) {
        const int64_t slot = w * GPW + grp;
        const bool act = (grp < GPW) && (slot < n_rows);
        const int32_t i = act ? static_cast<int32_t>(slot) : 0;
        double s = 0.0;
        if (act) s = block_row_dot<MT, BS, true>(A, vals, z, ii, A.diag[i] + 1, A.row_ptr[i + 1], 0.0);
        double b[BS];
#pragma unroll
        for (int j = 0; j < BS; ++j) b[j] = __shfl_sync(0xffffffffu, s, base + j);
        double zi = 0.0;
        if (act) {
            const MT* di = dinv + int64_t(i) * (BS * BS) + ii * BS;
            double x = 0.0;
#pragma unroll
            for (int j = 0; j < BS; ++j) x += ld(di + j) * b[j];
            zi = z[int64_t(i) * BS + ii] + x;
            z[int64_t(i) * BS + ii] = zi;
        }
        double zr[BS];
#pragma unroll
        for (int j = 0; j < BS; ++j) zr[j] = __shfl_sync(0xffffffffu, zi, base + j);
        if (act) {
            const MT* ad = vals + int64_t(A.diag[i]) * (BS * BS) + ii * BS;
            double d = 0.0;
#pragma unroll
            for (int jj = 0; jj < BS; ++jj) d += ld(ad + jj) * zr[jj];
            const double yv = d - s;
            const int64_t t = int64_t(i) * BS + ii;
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
    if constexpr (ND > 0) block_reduce_store<ND, 256>(pr, partials + size_t(blockIdx.x) * ND);
}

// ------------------------------------------------------ Krylov kernels
// r = b - v, r0 = r, p = r; partial sums of |b|^2 and |r|^2.
__global__ void __launch_bounds__(kVecThreads) k_krylov_init(int64_t len, const double* __restrict__ b,
                                                             const double* __restrict__ v, double* __restrict__ r,
                                                             double* __restrict__ r0, double* __restrict__ p,
                                                             double* __restrict__ partials) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    double pr[2] = {0.0, 0.0};
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < len; t += stride) {
        const double bt = b[t];
        const double rt = bt + (-1.0) * v[t];
        r[t] = rt;
        r0[t] = rt;
        p[t] = rt;
        pr[0] += bt * bt;
        pr[1] += rt * rt;
    }
    block_reduce_store<2, kVecThreads>(pr, partials + size_t(blockIdx.x) * 2);
}

// Sum of column k of the per-block partials (stride values per block) by the
// whole block: thread t adds blocks t, t+T, ... in order, then a fixed-order
// tree; every thread returns the same total.  Deterministic for a given
// partial count.
constexpr int kFinThreads = 512;

__device__ __forceinline__ double block_sum_partials(const double* __restrict__ partials, int nblocks, int stride,
                                                     int k) {
    __shared__ double sh[kFinThreads / 32];
    __shared__ double total;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partials[size_t(b) * stride + k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = s;
    __syncthreads();
    if (warp == 0) {
        double x = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) total = x;
    }
    __syncthreads();
    const double r = total;
    __syncthreads();
    return r;
}

__global__ void k_krylov_init_fin(KrylovScalars* ks, const double* __restrict__ partials, int nblocks) {
    const double bnorm = sqrt(block_sum_partials(partials, nblocks, 2, 0));
    double rnorm = sqrt(block_sum_partials(partials, nblocks, 2, 1));
    if (threadIdx.x != 0) return;
    const double scale = (bnorm > 0.0) ? bnorm : 1.0;
    ks->bnorm = bnorm;
    ks->scale = scale;
    ks->tol = fmax(ks->abs_tol, ks->rel_tol * scale);
    double r0n = rnorm;
    if (ks->guess == 1 && !(rnorm < bnorm)) {  // the guess does not beat x = 0
        ks->guess = 2;
        r0n = bnorm;
    }
    rnorm = r0n;
    ks->initial = rnorm;
    ks->rnorm = rnorm;
    ks->it = 0;
    ks->state = KS_RUNNING;
    if (!isfinite(rnorm)) {
        ks->state = KS_DIVERGED;
    } else if (rnorm <= ks->tol) {
        ks->state = KS_CONVERGED;
    }
    ks->rho = rnorm * rnorm;
    ks->rho_old = 1.0;
    ks->alpha = 1.0;
    ks->omega = 1.0;
    ks->beta = 0.0;
}

// gamma = r0.v -> alpha = rho / gamma (bicgstab.cpp:112-119); also counts
// the iteration and stops at max_it.
__global__ void k_krylov_gamma(KrylovScalars* ks, const double* __restrict__ partials, int nblocks) {
    if (ks->state != KS_RUNNING) return;  // uniform
    const double gamma = block_sum_partials(partials, nblocks, 1, 0);
    if (threadIdx.x != 0) return;
    if (!isfinite(gamma) || gamma == 0.0) {
        ks->state = KS_DIVERGED;
        return;
    }
    ks->alpha = ks->rho / gamma;
}

// Iteration gate: stops at max_it before any work of iteration it+1,
// checks beta of the search direction update (bicgstab.cpp:88-104).
__global__ void k_krylov_begin(KrylovScalars* ks) {
    if (threadIdx.x != 0 || ks->state != KS_RUNNING) return;
    if (ks->it >= ks->max_it) {
        ks->state = KS_MAXIT;
        return;
    }
    ks->it += 1;
    if (ks->it > 1 && !isfinite(ks->beta)) ks->state = KS_DIVERGED;
}

// s = r - alpha v
__global__ void __launch_bounds__(kVecThreads) k_krylov_s(int64_t len, const KrylovScalars* __restrict__ ks,
                                                          const double* __restrict__ r, const double* __restrict__ v,
                                                          double* __restrict__ s) {
    if (ks->state != KS_RUNNING) return;
    const double alpha = ks->alpha;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < len; t += stride)
        s[t] = r[t] + (-alpha) * v[t];
}

// Five fused inner products -> omega, reconstructed |r|, rho_next
// (bicgstab.cpp:128-158), pre-update breakdown checks.
__global__ void k_krylov_omega(KrylovScalars* ks, const double* __restrict__ partials, int nblocks) {
    if (ks->state != KS_RUNNING) return;  // uniform
    const double tt = block_sum_partials(partials, nblocks, 5, 0);
    const double ts = block_sum_partials(partials, nblocks, 5, 1);
    const double r0t = block_sum_partials(partials, nblocks, 5, 2);
    const double r0s = block_sum_partials(partials, nblocks, 5, 3);
    const double ss = block_sum_partials(partials, nblocks, 5, 4);
    if (threadIdx.x != 0) return;
    if (!isfinite(ts) || !isfinite(tt) || tt == 0.0) {
        ks->state = KS_DIVERGED;
        return;
    }
    const double omega_new = ts / tt;
    const double rn2 = ss - 2.0 * omega_new * ts + omega_new * omega_new * tt;
    ks->omega_new = omega_new;
    ks->rnorm = sqrt(fmax(rn2, 0.0));
    ks->rho_new = r0s - omega_new * r0t;
    ks->beta = (ks->rho_new / ks->rho) * (ks->alpha / omega_new);
}

// x += alpha phat + omega shat; r = s - omega t; next p = r + beta (p - omega v);
// partial |r|^2 for the periodic true-norm refresh.
__global__ void __launch_bounds__(kVecThreads) k_krylov_update(int64_t len, const KrylovScalars* __restrict__ ks,
                                                               double* __restrict__ x, const double* __restrict__ phat,
                                                               const double* __restrict__ shat,
                                                               const double* __restrict__ s,
                                                               const double* __restrict__ tv, double* __restrict__ r,
                                                               double* __restrict__ p, const double* __restrict__ v,
                                                               double* __restrict__ partials) {
    if (ks->state != KS_RUNNING) return;  // uniform across the grid
    const double alpha = ks->alpha, omega = ks->omega_new, beta = ks->beta;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    double pr[1] = {0.0};
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < len; t += stride) {
        double xv = x[t] + alpha * phat[t];
        xv = xv + omega * shat[t];
        x[t] = xv;
        const double rv = s[t] + (-omega) * tv[t];
        r[t] = rv;
        double pv = beta * p[t];
        pv = pv + (-beta * omega) * v[t];
        pv = pv + 1.0 * rv;
        p[t] = pv;
        pr[0] += rv * rv;
    }
    block_reduce_store<1, kVecThreads>(pr, partials + size_t(blockIdx.x));
}

// Post-update checks, refresh every 32 iterations, convergence test
// (bicgstab.cpp:149-176).
__global__ void k_krylov_post(KrylovScalars* ks, const double* __restrict__ partials, int nblocks) {
    if (ks->state != KS_RUNNING) return;  // uniform
    const bool refresh = (ks->it % 32 == 0);
    const double rr = refresh ? block_sum_partials(partials, nblocks, 1, 0) : 0.0;
    if (threadIdx.x != 0) return;
    const double omega_new = ks->omega_new;
    double rnorm = ks->rnorm;
    if (!isfinite(rnorm) || !isfinite(omega_new) || omega_new == 0.0) {
        ks->state = KS_DIVERGED;
        return;
    }
    if (refresh) {
        rnorm = sqrt(rr);
        ks->rnorm = rnorm;
    }
    if (rnorm <= ks->tol) {
        ks->state = KS_CONVERGED;
        return;
    }
    if (!isfinite(ks->rho_new) || ks->rho_new == 0.0) {
        ks->state = KS_DIVERGED;
        return;
    }
    ks->rho_old = ks->rho;
    ks->rho = ks->rho_new;
    ks->omega = omega_new;
}

// The while-condition of the device loop.  body_runs grows by one per body
// run whatever the state, so the loop ends after at most max_it runs even if
// the state were never updated.
__global__ void k_krylov_cond(KrylovScalars* ks, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0) return;
    const int runs = ks->body_runs + 1;
    ks->body_runs = runs;
    const bool more = ks->state == KS_RUNNING && runs < ks->max_it;
    cudaGraphSetConditional(h, more ? 1u : 0u);
}

}  // namespace

// ------------------------------------------------------------- launchers
int spmv_blocks(int32_t n, int32_t bs) { return static_cast<int>(vec_grid(int64_t(n) * bs)); }

// One wave of the fused pass: its launch bounds let 6 (bs <= 5) or 5 (6x6)
// 256-thread blocks share an SM, so the grid-stride loop runs on exactly the
// resident blocks.
int sgs_last_spmv_blocks(int32_t n_rows, int32_t bs) {
    const int64_t warps = (int64_t(n_rows) + (32 / bs) - 1) / (32 / bs);
    const int64_t g = (warps + 7) / 8;
    const int64_t cap = int64_t(148) * (bs <= 5 ? 6 : 5);
    return static_cast<int>(g < 1 ? 1 : (g < cap ? g : cap));
}

template <typename MT>
void launch_sgs_last_spmv(const BsrView& A, const MT* vals, const MT* dinv, int32_t n_rows, double* z, double* y,
                          const DotSpec& ds, double* partials, const int* active, cudaStream_t s) {
    const unsigned gr = static_cast<unsigned>(sgs_last_spmv_blocks(n_rows, A.bs));
#define CFDG_FUSED(BS)                                                                                     \
    if (ds.n == 0) k_sgs_last_spmv<MT, BS, 0><<<gr, 256, 0, s>>>(A, vals, dinv, n_rows, z, y, ds, partials, active); \
    else if (ds.n == 1) k_sgs_last_spmv<MT, BS, 1><<<gr, 256, 0, s>>>(A, vals, dinv, n_rows, z, y, ds, partials, active); \
    else k_sgs_last_spmv<MT, BS, 5><<<gr, 256, 0, s>>>(A, vals, dinv, n_rows, z, y, ds, partials, active)
    switch (A.bs) {
        case 1: CFDG_FUSED(1); break;
        case 3: CFDG_FUSED(3); break;
        case 4: CFDG_FUSED(4); break;
        case 5: CFDG_FUSED(5); break;
        case 6: CFDG_FUSED(6); break;
        default: break;
    }
#undef CFDG_FUSED
}

template <typename MT>
void launch_spmv_ex(const BsrView& A, const MT* vals, const double* x, double* y, double alpha, double beta,
                    const DotSpec& ds, double* partials, const int* active, cudaStream_t s, int32_t row_begin) {
    const unsigned gr = vec_grid(int64_t(A.n - row_begin) * A.bs);
    const int nd = ds.n;
#define CFDG_SPMV(BS, ND) \
    k_spmv<MT, BS, ND><<<gr, kVecThreads, 0, s>>>(A, vals, x, y, alpha, beta, ds, partials, active, row_begin)
    if (A.bs == 5) {
        if (nd == 0) CFDG_SPMV(5, 0);
        else if (nd == 1) CFDG_SPMV(5, 1);
        else CFDG_SPMV(5, 5);
    } else if (A.bs == 6) {
        if (nd == 0) CFDG_SPMV(6, 0);
        else if (nd == 1) CFDG_SPMV(6, 1);
        else CFDG_SPMV(6, 5);
    } else if (A.bs == 1) {
        if (nd == 0) CFDG_SPMV(1, 0);
        else if (nd == 1) CFDG_SPMV(1, 1);
        else CFDG_SPMV(1, 5);
    } else if (A.bs == 3) {
        if (nd == 0) CFDG_SPMV(3, 0);
        else if (nd == 1) CFDG_SPMV(3, 1);
        else CFDG_SPMV(3, 5);
    } else if (A.bs == 4) {
        if (nd == 0) CFDG_SPMV(4, 0);
        else if (nd == 1) CFDG_SPMV(4, 1);
        else CFDG_SPMV(4, 5);
    }
#undef CFDG_SPMV
}

template <typename MT>
void launch_lu_setup(const BsrView& A, const MT* vals, MT* lu, int8_t* piv, int* err_flag, bool inverse,
                     cudaStream_t s) {
    const unsigned gr = grid_for(A.n, kLuThreads);
#define CFDG_LU(BS)                                                                          \
    if (inverse) k_lu<MT, BS, true><<<gr, kLuThreads, 0, s>>>(A, vals, lu, piv, err_flag); \
    else k_lu<MT, BS, false><<<gr, kLuThreads, 0, s>>>(A, vals, lu, piv, err_flag)
    switch (A.bs) {
        case 1: CFDG_LU(1); break;
        case 3: CFDG_LU(3); break;
        case 4: CFDG_LU(4); break;
        case 5: CFDG_LU(5); break;
        case 6: CFDG_LU(6); break;
        default: break;
    }
#undef CFDG_LU
}

template <typename MT>
void launch_sgs_rows_ex(const BsrView& A, const MT* vals, const MT* lu, const int8_t* piv, const int32_t* rows,
                        int32_t row0, int32_t n_rows, const double* r, double* z, int mode, bool inverse,
                        const int* active, cudaStream_t s) {
    if (n_rows <= 0) return;
    const int gpw = 32 / A.bs;
    const int64_t warps = (int64_t(n_rows) + gpw - 1) / gpw;
    const unsigned gr = grid_for(warps * 32, 256);
#define CFDG_SGS_M(BS, M)                                                                                      \
    if (inverse) k_sgs_rows<MT, BS, M, true><<<gr, 256, 0, s>>>(A, vals, lu, piv, rows, row0, n_rows, r, z, active); \
    else k_sgs_rows<MT, BS, M, false><<<gr, 256, 0, s>>>(A, vals, lu, piv, rows, row0, n_rows, r, z, active)
#define CFDG_SGS(BS)                           \
    if (mode == 0) { CFDG_SGS_M(BS, 0); }      \
    else if (mode == 1) { CFDG_SGS_M(BS, 1); } \
    else if (mode == 2) { CFDG_SGS_M(BS, 2); } \
    else { CFDG_SGS_M(BS, 3); }
    switch (A.bs) {
        case 1: CFDG_SGS(1); break;
        case 3: CFDG_SGS(3); break;
        case 4: CFDG_SGS(4); break;
        case 5: CFDG_SGS(5); break;
        case 6: CFDG_SGS(6); break;
        default: break;
    }
#undef CFDG_SGS
#undef CFDG_SGS_M
}

// Resident 256-thread blocks of the cooperative sweep on the current device
// (at most 4 per SM), 0 without cooperative launch; cached per device.
template <typename MT, int BS>
static int level_coop_grid() {
    constexpr int kMaxDevices = 64;
    static std::atomic<int> cache[kMaxDevices];  // 0: unknown, -1: unavailable, else the grid
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return 0;
    }
    int grid = cache[dev].load();
    if (grid == 0) {
        int sms = 0, per_sm = 0, coop = 0;
        grid = -1;
        if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) == cudaSuccess && coop &&
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sgs_level_coop<MT, BS>, 256, 0) == cudaSuccess &&
            per_sm > 0)
            grid = sms * std::min(per_sm, 4);
        cudaGetLastError();
        cache[dev].store(grid);
    }
    return grid > 0 ? grid : 0;
}

template <typename MT>
bool launch_sgs_level_coop(const BsrView& A, const MT* vals, const MT* lu, const int8_t* piv, const int4* fwd_rows,
                           const int32_t* fwd_off, int n_fwd, const int4* bwd_rows, const int32_t* bwd_off,
                           int n_bwd, const double* r, double* z, const int* active, cudaStream_t s) {
    void* args[] = {const_cast<BsrView*>(&A), &vals, &lu, &piv, &fwd_rows, &fwd_off, &n_fwd, &bwd_rows, &bwd_off,
                    &n_bwd, &r, &z, &active};
    int grid = 0;
    void* fn = nullptr;
    switch (A.bs) {
        case 5: grid = level_coop_grid<MT, 5>(); fn = reinterpret_cast<void*>(k_sgs_level_coop<MT, 5>); break;
        case 6: grid = level_coop_grid<MT, 6>(); fn = reinterpret_cast<void*>(k_sgs_level_coop<MT, 6>); break;
        default: return false;
    }
    if (grid <= 0) return false;
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(256), args, 0, s) == cudaSuccess;
}

int dot_blocks(int64_t len) { return static_cast<int>(vec_grid(len)); }

void launch_krylov_init(int64_t len, const double* b, const double* v, double* r, double* r0, double* p,
                        double* partials, KrylovScalars* ks, cudaStream_t s) {
    const unsigned gr = vec_grid(len);
    k_krylov_init<<<gr, kVecThreads, 0, s>>>(len, b, v, r, r0, p, partials);
    k_krylov_init_fin<<<1, kFinThreads, 0, s>>>(ks, partials, static_cast<int>(gr));
}
__global__ void __launch_bounds__(kVecThreads) k_krylov_guess_reset(int64_t len, const KrylovScalars* __restrict__ ks,
                                                                    const double* __restrict__ b, double* __restrict__ x,
                                                                    double* __restrict__ r, double* __restrict__ r0,
                                                                    double* __restrict__ p) {
    if (ks->guess != 2) return;  // uniform
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; t < len; t += stride) {
        const double bt = b[t];
        x[t] = 0.0;
        r[t] = bt;
        r0[t] = bt;
        p[t] = bt;
    }
}

void launch_krylov_guess_reset(int64_t len, const KrylovScalars* ks, const double* b, double* x, double* r, double* r0,
                               double* p, cudaStream_t s) {
    k_krylov_guess_reset<<<vec_grid(len), kVecThreads, 0, s>>>(len, ks, b, x, r, r0, p);
}

void launch_krylov_begin(KrylovScalars* ks, cudaStream_t s) { k_krylov_begin<<<1, 32, 0, s>>>(ks); }
void launch_krylov_gamma(KrylovScalars* ks, const double* partials, int nblocks, cudaStream_t s) {
    k_krylov_gamma<<<1, kFinThreads, 0, s>>>(ks, partials, nblocks);
}
void launch_krylov_s(int64_t len, const KrylovScalars* ks, const double* r, const double* v, double* sv,
                     cudaStream_t s) {
    k_krylov_s<<<vec_grid(len), kVecThreads, 0, s>>>(len, ks, r, v, sv);
}
void launch_krylov_omega(KrylovScalars* ks, const double* partials, int nblocks, cudaStream_t s) {
    k_krylov_omega<<<1, kFinThreads, 0, s>>>(ks, partials, nblocks);
}
void launch_krylov_update(int64_t len, const KrylovScalars* ks, double* x, const double* phat, const double* shat,
                          const double* sv, const double* tv, double* r, double* p, const double* v,
                          double* partials, cudaStream_t s) {
    k_krylov_update<<<vec_grid(len), kVecThreads, 0, s>>>(len, ks, x, phat, shat, sv, tv, r, p, v, partials);
}
void launch_krylov_post(KrylovScalars* ks, const double* partials, int nblocks, cudaStream_t s) {
    k_krylov_post<<<1, kFinThreads, 0, s>>>(ks, partials, nblocks);
}

template void launch_spmv_ex<double>(const BsrView&, const double*, const double*, double*, double, double,
                                     const DotSpec&, double*, const int*, cudaStream_t, int32_t);
template void launch_spmv_ex<float>(const BsrView&, const float*, const double*, double*, double, double,
                                    const DotSpec&, double*, const int*, cudaStream_t, int32_t);
template void launch_sgs_last_spmv<double>(const BsrView&, const double*, const double*, int32_t, double*, double*,
                                           const DotSpec&, double*, const int*, cudaStream_t);
template void launch_sgs_last_spmv<float>(const BsrView&, const float*, const float*, int32_t, double*, double*,
                                          const DotSpec&, double*, const int*, cudaStream_t);
template void launch_lu_setup<double>(const BsrView&, const double*, double*, int8_t*, int*, bool, cudaStream_t);
template void launch_lu_setup<float>(const BsrView&, const float*, float*, int8_t*, int*, bool, cudaStream_t);
template bool launch_sgs_level_coop<double>(const BsrView&, const double*, const double*, const int8_t*,
                                            const int4*, const int32_t*, int, const int4*, const int32_t*, int,
                                            const double*, double*, const int*, cudaStream_t);
template bool launch_sgs_level_coop<float>(const BsrView&, const float*, const float*, const int8_t*, const int4*,
                                           const int32_t*, int, const int4*, const int32_t*, int, const double*,
                                           double*, const int*, cudaStream_t);
template void launch_sgs_rows_ex<double>(const BsrView&, const double*, const double*, const int8_t*, const int32_t*,
                                         int32_t, int32_t, const double*, double*, int, bool, const int*,
                                         cudaStream_t);
template void launch_sgs_rows_ex<float>(const BsrView&, const float*, const float*, const int8_t*, const int32_t*,
                                        int32_t, int32_t, const double*, double*, int, bool, const int*,
                                        cudaStream_t);

void launch_krylov_cond(KrylovScalars* ks, cudaGraphConditionalHandle h, cudaStream_t s) {
    k_krylov_cond<<<1, 32, 0, s>>>(ks, h);
}

}  // namespace cfdg
