// First-order Picard Jacobian assembly into BSR (JacobianKernel::apply,
// include/cfd/solver/compressible/jacobian_kernel.hpp:74-270).
//
// Every off-diagonal block belongs to exactly one interior face, so the face
// kernel writes it directly at a position precomputed on the host (no
// binary search, no atomics):  A(c0,c1) = dF/dUR,  A(c1,c0) = -dF/dUL.
// The diagonal block of cell c is the sum of the owner-side contributions of
// its faces, which are minus the transposed off-diagonal blocks, plus the
// boundary-face blocks and alpha*I; the diagonal kernel gathers them in the
// same order as the sequential reference adds them.
#include "cfdg.h"
#include "kernels.hpp"
#include "physics.cuh"

namespace cfdg {

namespace {

template <typename MT>
__device__ __forceinline__ MT to_mt(double x) { return static_cast<MT>(x); }

// dF/dU of one side: A*(0.5*J(U) + sgn*0.5*smax*I) (+ viscous, sign vs),
// HllcFlux::face_flux_jacobian (fluxes/hllc.hpp:135-168),
// ViscousFlux::face_flux_jacobian (fluxes/viscous.hpp:280-360).
__device__ __forceinline__ void side_jacobian(const GasParams& g, const double U[5], double nx, double ny, double nz,
                                              double half_area, double diss, double J[25]) {
    euler_jacobian(g, U, nx, ny, nz, J);
#pragma unroll
    for (int i = 0; i < 25; ++i) J[i] *= half_area;
#pragma unroll
    for (int i = 0; i < 5; ++i) J[i * 6] += diss;
}

// Stores the block each lane of the warp holds in `stage[lane]` to its BSR
// slot: the warp walks its 32 faces and writes one contiguous block per step
// (coalesced), instead of 32 scattered 8-byte stores per instruction.
template <typename MT, int BS>
__device__ __forceinline__ void warp_store_blocks(MT (*stage)[BS * BS], int32_t pos, bool valid, MT* vals) {
    __syncwarp();
    const int lane = threadIdx.x & 31;
    for (int src = 0; src < 32; ++src) {
        const int32_t p = __shfl_sync(0xffffffffu, pos, src);
        const int ok = __shfl_sync(0xffffffffu, valid ? 1 : 0, src);
        if (!ok) continue;
        MT* dst = vals + int64_t(p) * (BS * BS);
        for (int e = lane; e < BS * BS; e += 32) dst[e] = stage[src][e];
    }
    __syncwarp();
}

template <typename MT, bool VISC, int BS, bool FULL>
__global__ void __launch_bounds__(128) k_jac_offdiag(DevMesh m, DevFields f, GasParams g, JacStructure js, MT* vals) {
    __shared__ MT stage_all[4][32][BS * BS];
    MT(*stage)[BS * BS] = stage_all[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int32_t fc = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = fc < m.ni;
    const int32_t fcs = valid ? fc : 0;  // lanes past the end compute on face 0 and store nothing
    const int64_t nt = m.nt;
    const int32_t c0 = m.owner[fcs], c1 = m.neigh[fcs];
    const double nx = m.fnx[fcs], ny = m.fny[fcs], nz = m.fnz[fcs], A = m.farea[fcs];
    double qL[5], qR[5], UL[5], UR[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        qL[v] = f.q[v * nt + c0];
        qR[v] = f.q[v * nt + c1];
    }
    prim_to_cons(g, qL[0], qL[1], qL[2], qL[3], qL[4], UL);
    prim_to_cons(g, qR[0], qR[1], qR[2], qR[3], qR[4], UR);
    const double smax = hllc_smax(g, UL, UR, nx, ny, nz);
    const double half_area = 0.5 * A, diss = 0.5 * smax * A;
    double mutL = 0.0, mutR = 0.0;
    if (VISC && f.mut) {
        mutL = f.mut[c0];
        mutR = f.mut[c1];
    }
    double J[25];
    // A(c0, c1) += dF/dUR
    side_jacobian(g, UR, nx, ny, nz, half_area, -diss, J);
    if (VISC) viscous_jacobian_add<FULL>(g, m.finv_d[fcs], qL, qR, mutL, mutR, A, -1.0, J, nx, ny, nz);
#pragma unroll
    for (int r = 0; r < BS; ++r)
#pragma unroll
        for (int c = 0; c < BS; ++c) stage[lane][r * BS + c] = (r < 5 && c < 5) ? to_mt<MT>(J[r * 5 + c]) : MT(0);
    // nu_tilde entry of A(c0, c1): d F_nu / d (rho nu_tilde)_R (Picard: no coupling)
    if (BS == 6) stage[lane][35] = to_mt<MT>(js.sa_jac[m.nf + fcs]);
    warp_store_blocks<MT, BS>(stage, js.face_pos[2 * fcs], valid, vals);
    // A(c1, c0) -= dF/dUL
    side_jacobian(g, UL, nx, ny, nz, half_area, diss, J);
    if (VISC) viscous_jacobian_add<FULL>(g, m.finv_d[fcs], qL, qR, mutL, mutR, A, 1.0, J, nx, ny, nz);
#pragma unroll
    for (int r = 0; r < BS; ++r)
#pragma unroll
        for (int c = 0; c < BS; ++c) stage[lane][r * BS + c] = (r < 5 && c < 5) ? to_mt<MT>(-J[r * 5 + c]) : MT(0);
    if (BS == 6) stage[lane][35] = to_mt<MT>(-js.sa_jac[fcs]);  // A(c1, c0) -= d F_nu / d (rho nu_tilde)_L
    warp_store_blocks<MT, BS>(stage, js.face_pos[2 * fcs + 1], valid, vals);
}

// Boundary faces: owner-side block only, first-order states against the BC
// ghost, ghost eddy viscosity zero (jacobian_kernel.hpp:232-269).  FULL:
// the no-slip ghost's mirrored velocity (and isothermal temperature) doubles
// the owner's viscous derivative.
template <bool VISC, bool FULL>
__global__ void __launch_bounds__(128) k_jac_bface(DevMesh m, DevFields f, GasParams g, double* __restrict__ out) {
    const int32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= m.nb) return;
    const int64_t nt = m.nt;
    const int32_t fc = m.ni + b;
    const int32_t c0 = m.owner[fc];
    const int64_t cg = int64_t(m.n) + b;
    const double nx = m.fnx[fc], ny = m.fny[fc], nz = m.fnz[fc], A = m.farea[fc];
    double qL[5], qR[5], UL[5], UR[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        qL[v] = f.q[v * nt + c0];
        qR[v] = f.q[v * nt + cg];
    }
    prim_to_cons(g, qL[0], qL[1], qL[2], qL[3], qL[4], UL);
    prim_to_cons(g, qR[0], qR[1], qR[2], qR[3], qR[4], UR);
    const double smax = hllc_smax(g, UL, UR, nx, ny, nz);
    double J[25];
    side_jacobian(g, UL, nx, ny, nz, 0.5 * A, 0.5 * smax * A, J);
    if (VISC) {
        const double mutL = f.mut ? f.mut[c0] : 0.0;
        const int kind = m.patches[m.bpatch[b]].kind;
        const bool noslip = kind == CFDG_BC_NO_SLIP_WALL || kind == CFDG_BC_NO_SLIP_WALL_HEAT_FLUX;
        const double wv = noslip ? 2.0 : 1.0, wt = kind == CFDG_BC_NO_SLIP_WALL ? 2.0 : 1.0;
        viscous_jacobian_add<FULL>(g, m.finv_d[fc], qL, qR, mutL, 0.0, A, 1.0, J, nx, ny, nz, wv, wt);
    }
#pragma unroll
    for (int i = 0; i < 25; ++i) out[int64_t(b) * 25 + i] = J[i];
}

// Diagonal block entry (c, e): -sum of transposed off-diagonal blocks of row
// c, + boundary-face blocks, + alpha on the diagonal.  With 6x6 blocks the
// nu_tilde row and column are zero except [5][5] = -sum of the transposed
// [5][5] entries + the boundary faces' d F_nu / d (rho nu_tilde) + the
// destruction derivative + alpha (Picard: no mean-flow coupling).
template <typename MT, int BS>
__global__ void __launch_bounds__(256) k_jac_diag(DevMesh m, const double* __restrict__ alpha, JacStructure js,
                                                  const double* __restrict__ bjac, MT* vals) {
    constexpr int NE = BS * BS;
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(m.n) * NE) return;
    const int32_t c = static_cast<int32_t>(t / NE);
    const int32_t row = row_index(m, c);
    const int eb = static_cast<int>(t % NE);
    const int er = eb / BS, ec = eb % BS;
    const int32_t d = js.diag[row];
    double v = 0.0;
    if (er < 5 && ec < 5) {
        const int e = er * 5 + ec;
        for (int32_t k = js.row_ptr[row]; k < js.row_ptr[row + 1]; ++k) {
            if (k == d) continue;
            v -= static_cast<double>(vals[int64_t(js.trans[k]) * NE + eb]);
        }
        for (int32_t q = m.c2f_off[c]; q < m.c2f_off[c + 1]; ++q) {
            const int32_t fc = m.c2f[q];
            if (fc >= m.ni) v += bjac[int64_t(fc - m.ni) * 25 + e];
        }
        if (er == ec && alpha) v += alpha[c];
    } else if (er == 5 && ec == 5) {
        for (int32_t k = js.row_ptr[row]; k < js.row_ptr[row + 1]; ++k) {
            if (k == d) continue;
            v -= static_cast<double>(vals[int64_t(js.trans[k]) * NE + eb]);
        }
        for (int32_t q = m.c2f_off[c]; q < m.c2f_off[c + 1]; ++q) {
            const int32_t fc = m.c2f[q];
            if (fc >= m.ni) v += js.sa_jac[fc];
        }
        v += js.sa_dsrc[c] + alpha[c];
    }
    vals[int64_t(d) * NE + eb] = to_mt<MT>(v);
}

}  // namespace

template <typename MT, bool FULL>
static void launch_jacobian_t(const DevMesh& m, const DevFields& f, const GasParams& g, const JacStructure& js, int bs,
                              bool visc, MT* values, double* bface_scratch, cudaStream_t s) {
    if (m.ni > 0) {
        const unsigned gr = grid_for(m.ni, 128);
        if (bs == 5) {
            if (visc) k_jac_offdiag<MT, true, 5, FULL><<<gr, 128, 0, s>>>(m, f, g, js, values);
            else k_jac_offdiag<MT, false, 5, FULL><<<gr, 128, 0, s>>>(m, f, g, js, values);
        } else {
            if (visc) k_jac_offdiag<MT, true, 6, FULL><<<gr, 128, 0, s>>>(m, f, g, js, values);
            else k_jac_offdiag<MT, false, 6, FULL><<<gr, 128, 0, s>>>(m, f, g, js, values);
        }
    }
    if (m.nb > 0) {
        const unsigned gr = grid_for(m.nb, 128);
        if (visc) k_jac_bface<true, FULL><<<gr, 128, 0, s>>>(m, f, g, bface_scratch);
        else k_jac_bface<false, FULL><<<gr, 128, 0, s>>>(m, f, g, bface_scratch);
    }
    if (bs == 5) k_jac_diag<MT, 5><<<grid_for(int64_t(m.n) * 25, 256), 256, 0, s>>>(m, f.alpha, js, bface_scratch, values);
    else k_jac_diag<MT, 6><<<grid_for(int64_t(m.n) * 36, 256), 256, 0, s>>>(m, f.alpha, js, bface_scratch, values);
}

template <typename MT>
void launch_jacobian(const DevMesh& m, const DevFields& f, const GasParams& g, const JacStructure& js, int bs,
                     bool visc, MT* values, double* bface_scratch, cudaStream_t s) {
    if (js.full_viscous && visc) launch_jacobian_t<MT, true>(m, f, g, js, bs, visc, values, bface_scratch, s);
    else launch_jacobian_t<MT, false>(m, f, g, js, bs, visc, values, bface_scratch, s);
}

template void launch_jacobian<double>(const DevMesh&, const DevFields&, const GasParams&, const JacStructure&, int,
                                      bool, double*, double*, cudaStream_t);
template void launch_jacobian<float>(const DevMesh&, const DevFields&, const GasParams&, const JacStructure&, int,
                                     bool, float*, double*, cudaStream_t);

}  // namespace cfdg
