// First-order Picard Jacobian assembly into BSR (JacobianKernel::apply,
// include/cfd/solver/compressible/jacobian_kernel.hpp:74-270).
//
// Row-centric: one thread per block row (cell) walks the cell's faces in
// ascending face order, as the sequential reference does, and for each
// interior face writes the off-diagonal block of its row,
//   A(owner, neigh) = dF/dU_R  or  A(neigh, owner) = -dF/dU_L,
// while it accumulates its own side's contribution into the diagonal block
// (+dF/dU_L as owner, -dF/dU_R as neighbour, + the boundary faces' dF/dU_L,
// then alpha*I) in the reference's order.  Each block is written once, the
// rows of a warp are consecutive so its stores cover one contiguous range,
// and no block is read back to form the diagonal.
#include "cfdg.h"
#include "kernels.hpp"
#include "physics.cuh"

namespace cfdg {

namespace {

template <typename MT>
__device__ __forceinline__ MT to_mt(double x) { return static_cast<MT>(x); }

// Stores the block each lane of the warp holds in `stage[lane]` to its BSR
// slot: the warp walks its 32 lanes' blocks and writes one contiguous block
// per step (coalesced), instead of 32 scattered stores per instruction.
// Staged block row stride: BS*BS padded to an odd number of elements so
// that the 32 lanes writing entry e of their own block hit distinct banks.
template <int BS>
__host__ __device__ constexpr int stage_stride() { return (BS * BS) % 2 == 0 ? BS * BS + 1 : BS * BS; }

template <typename MT, int BS>
__device__ __forceinline__ void warp_store_blocks(MT (*stage)[stage_stride<BS>()], int32_t pos, bool valid,
                                                  MT* vals) {
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

// Entry-wise restatement of side_jacobian + viscous_jacobian_add (same
// expressions, same rounding sequence per entry: Euler entry * A/2, + the
// dissipation on the diagonal, + s * viscous entry), so that a block is
// produced one entry at a time straight into its destination instead of as
// a 25-double array per side.
struct EulerState {
    double u, v, w, H, hpq, phi, gamma;
};
__device__ __forceinline__ EulerState euler_state(const GasParams& g, const double U[5]) {
    EulerState e;
    const double rho = U[0];
    const double inv_rho = 1.0 / rho;
    e.u = U[1] * inv_rho;
    e.v = U[2] * inv_rho;
    e.w = U[3] * inv_rho;
    const double E = U[4] * inv_rho;
    const double p = pressure_of(g, U);
    e.gamma = g.gamma;
    e.phi = g.gamma - 1.0;
    const double q2 = e.u * e.u + e.v * e.v + e.w * e.w;
    e.H = E + p * inv_rho;
    e.hpq = 0.5 * e.phi * q2;
    return e;
}
// Entry (r, c) of the normal Euler flux Jacobian (euler_jacobian).
__device__ __forceinline__ double euler_entry(const EulerState& e, double nx, double ny, double nz, double un, int r,
                                              int c) {
    const double n[3] = {nx, ny, nz}, vel[3] = {e.u, e.v, e.w};
    if (r == 0) return (c >= 1 && c <= 3) ? n[c - 1] : 0.0;
    if (r == 4) {
        if (c == 0) return un * (e.hpq - e.H);
        if (c == 4) return e.gamma * un;
        return e.H * n[c - 1] - e.phi * vel[c - 1] * un;
    }
    const int a = r - 1;  // momentum component
    if (c == 0) return e.hpq * n[a] - vel[a] * un;
    if (c == 4) return e.phi * n[a];
    const int b = c - 1;
    if (a == b) return un + n[a] * (1.0 - e.phi) * vel[a];
    return vel[a] * n[b] - e.phi * n[a] * vel[b];
}

// Face quantities of the thin-layer viscous Jacobian (viscous_jacobian_add).
struct ViscFace {
    double u_f, v_f, w_f, T_f, inv_rho, inv_rho_cv, C_mu, C_lam, V2, cm, cl, Mu[3], uMu;
};
template <bool FULL>
__device__ __forceinline__ ViscFace visc_face(const GasParams& g, double inv_d, const double qL[5], const double qR[5],
                                              double mutL, double mutR, double area, double nx, double ny, double nz,
                                              double wv, double wt) {
    ViscFace v;
    const double p_f = 0.5 * (qL[0] + qR[0]);
    v.u_f = 0.5 * (qL[1] + qR[1]);
    v.v_f = 0.5 * (qL[2] + qR[2]);
    v.w_f = 0.5 * (qL[3] + qR[3]);
    v.T_f = 0.5 * (qL[4] + qR[4]);
    const double rho_f = p_f / (g.R * v.T_f);
    v.inv_rho = 1.0 / rho_f;
    v.inv_rho_cv = 1.0 / (rho_f * g.cv);
    const double mu_lam = sutherland(v.T_f);
    const double mu_t_f = 0.5 * (mutL + mutR);
    const double mu_eff = mu_lam + mu_t_f;
    const double k_lam = (mu_lam * g.cp) / g.prandtl;
    const double k_eff = k_lam + (mu_t_f * g.cp) / g.prandtl_turb;
    v.C_mu = mu_eff * inv_d * area;
    v.C_lam = k_eff * inv_d * area;
    v.V2 = v.u_f * v.u_f + v.v_f * v.v_f + v.w_f * v.w_f;
    v.cm = wv * v.C_mu;
    v.cl = wt * v.C_lam;
    v.uMu = 0.0;
    if (FULL) {
        const double un3 = (nx * v.u_f + ny * v.v_f + nz * v.w_f) * (1.0 / 3.0);
        v.Mu[0] = v.u_f + nx * un3;
        v.Mu[1] = v.v_f + ny * un3;
        v.Mu[2] = v.w_f + nz * un3;
        v.uMu = v.u_f * v.Mu[0] + v.v_f * v.Mu[1] + v.w_f * v.Mu[2];
    }
    return v;
}
// Entry (r, c) of the viscous Jacobian before the factor s.
template <bool FULL>
__device__ __forceinline__ double visc_entry(const ViscFace& v, const GasParams& g, double nx, double ny, double nz,
                                             int r, int c) {
    const double u[3] = {v.u_f, v.v_f, v.w_f};
    if (r == 0) return 0.0;
    if (!FULL) {
        if (r <= 3) {
            if (c == 0) return -v.C_mu * u[r - 1] * v.inv_rho;
            if (c == r) return v.C_mu * v.inv_rho;
            return 0.0;
        }
        if (c == 0) return v.C_lam * (0.5 * v.V2 - g.cv * v.T_f) * v.inv_rho_cv - v.C_mu * v.V2 * v.inv_rho;
        if (c == 4) return v.C_lam * v.inv_rho_cv;
        return -v.C_lam * u[c - 1] * v.inv_rho_cv + v.C_mu * u[c - 1] * v.inv_rho;
    }
    const double n[3] = {nx, ny, nz};
    if (r <= 3) {
        const int a = r - 1;
        if (c == 0) return -v.cm * v.Mu[a] * v.inv_rho;
        if (c == 4) return 0.0;
        const int b = c - 1;
        return v.cm * ((a == b ? 1.0 : 0.0) + n[a] * n[b] * (1.0 / 3.0)) * v.inv_rho;
    }
    if (c == 0) return v.cl * (0.5 * v.V2 - g.cv * v.T_f) * v.inv_rho_cv - v.cm * v.uMu * v.inv_rho;
    if (c == 4) return v.cl * v.inv_rho_cv;
    return -v.cl * u[c - 1] * v.inv_rho_cv + v.cm * v.Mu[c - 1] * v.inv_rho;
}

// 4 blocks of 128 threads per SM (128 registers), 3 for the viscous rows,
// whose per-thread state (the viscous face terms on top of the Euler
// ones) spills at 128 registers.
template <typename MT, bool VISC, int BS, bool FULL>
__global__ void __launch_bounds__(128, VISC ? 3 : 4)
    k_jac_rows(DevMesh m, DevFields f, GasParams g, JacStructure js, MT* vals) {
    __shared__ MT stage_all[4][32][stage_stride<BS>()];
    MT(*stage)[stage_stride<BS>()] = stage_all[threadIdx.x >> 5];
    const int lane = threadIdx.x & 31;
    const int32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = r < m.n;
    const int32_t rs = valid ? r : 0;
    const int32_t c = js.cell_of ? js.cell_of[rs] : rs;
    const int64_t nt = m.nt;
    double qc[5], Uc[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) qc[v] = f.q[v * nt + c];
    prim_to_cons(g, qc[0], qc[1], qc[2], qc[3], qc[4], Uc);
    const EulerState ec = euler_state(g, Uc);
    const double mutc = (VISC && f.mut) ? f.mut[c] : 0.0;
    double D[25];
#pragma unroll
    for (int i = 0; i < 25; ++i) D[i] = 0.0;
    double d35 = 0.0;
    const int32_t e0 = m.c2f_off[c];
    const int nfc = valid ? m.c2f_off[c + 1] - e0 : 0;
    const int maxf = __reduce_max_sync(0xffffffffu, nfc);
    for (int q = 0; q < maxf; ++q) {
        const bool has = q < nfc;
        const int32_t fc = has ? m.c2f[e0 + q] : 0;
        const bool inner = has && fc < m.ni;
        const double nx = m.fnx[fc], ny = m.fny[fc], nz = m.fnz[fc], A = m.farea[fc];
        const double half = 0.5 * A;
        const double unc = ec.u * nx + ec.v * ny + ec.w * nz;
        int32_t pos = 0;
        if (inner) {
            const int32_t o = m.owner[fc], nb = m.neigh[fc];
            const bool own = o == c;
            const int32_t j = own ? nb : o;
            double qj[5], Uj[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) qj[v] = f.q[v * nt + j];
            prim_to_cons(g, qj[0], qj[1], qj[2], qj[3], qj[4], Uj);
            const double* qL = own ? qc : qj;
            const double* qR = own ? qj : qc;
            const double smax = own ? hllc_smax(g, Uc, Uj, nx, ny, nz) : hllc_smax(g, Uj, Uc, nx, ny, nz);
            const double diss = 0.5 * smax * A;
            double mutL = 0.0, mutR = 0.0;
            if (VISC && f.mut) {
                mutL = own ? mutc : f.mut[j];
                mutR = own ? f.mut[j] : mutc;
            }
            ViscFace vf{};
            if (VISC) vf = visc_face<FULL>(g, m.finv_d[fc], qL, qR, mutL, mutR, A, nx, ny, nz, 1.0, 1.0);
            const double sgn = own ? 1.0 : -1.0;
            const EulerState ej = euler_state(g, Uj);
            const double unj = ej.u * nx + ej.v * ny + ej.w * nz;
            // off-diagonal block: own -> A(c, j) = dF/dU_R, else A(c, j) = -dF/dU_L;
            // own side into the diagonal: += dF/dU_L as owner, -= dF/dU_R as neighbour
#pragma unroll
            for (int rr = 0; rr < 5; ++rr)
#pragma unroll
                for (int cc = 0; cc < 5; ++cc) {
                    double o1 = euler_entry(ej, nx, ny, nz, unj, rr, cc) * half;
                    double d1 = euler_entry(ec, nx, ny, nz, unc, rr, cc) * half;
                    if (rr == cc) {
                        o1 += -sgn * diss;
                        d1 += sgn * diss;
                    }
                    if (VISC) {
                        const double ve = visc_entry<FULL>(vf, g, nx, ny, nz, rr, cc);
                        o1 += -sgn * ve;
                        d1 += sgn * ve;
                    }
                    stage[lane][rr * BS + cc] = to_mt<MT>(sgn * o1);
                    if (own) D[rr * 5 + cc] += d1;
                    else D[rr * 5 + cc] -= d1;
                }
            if (BS == 6) {
#pragma unroll
                for (int k = 0; k < 5; ++k) {
                    stage[lane][k * BS + 5] = MT(0);
                    stage[lane][5 * BS + k] = MT(0);
                }
                const double2 sj = reinterpret_cast<const double2*>(js.sa_jac)[fc];  // owner, neighbour
                stage[lane][BS * BS - 1] = to_mt<MT>(own ? sj.y : -sj.x);
                d35 += own ? sj.x : -sj.y;
            }
            pos = js.face_pos[2 * fc + (own ? 0 : 1)];
        } else if (has) {
            // boundary face: owner side against the BC ghost, ghost eddy
            // viscosity zero (jacobian_kernel.hpp:232-269)
            const int64_t cg = int64_t(m.n) + (fc - m.ni);
            double qg[5], Ug[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) qg[v] = f.q[v * nt + cg];
            prim_to_cons(g, qg[0], qg[1], qg[2], qg[3], qg[4], Ug);
            const double diss = 0.5 * hllc_smax(g, Uc, Ug, nx, ny, nz) * A;
            ViscFace vf{};
            if (VISC) {
                const int kind = m.patches[m.bpatch[fc - m.ni]].kind;
                const bool noslip = kind == CFDG_BC_NO_SLIP_WALL || kind == CFDG_BC_NO_SLIP_WALL_HEAT_FLUX;
                const double wv = noslip ? 2.0 : 1.0, wt = kind == CFDG_BC_NO_SLIP_WALL ? 2.0 : 1.0;
                vf = visc_face<FULL>(g, m.finv_d[fc], qc, qg, mutc, 0.0, A, nx, ny, nz, wv, wt);
            }
#pragma unroll
            for (int rr = 0; rr < 5; ++rr)
#pragma unroll
                for (int cc = 0; cc < 5; ++cc) {
                    double d1 = euler_entry(ec, nx, ny, nz, unc, rr, cc) * half;
                    if (rr == cc) d1 += diss;
                    if (VISC) d1 += visc_entry<FULL>(vf, g, nx, ny, nz, rr, cc);
                    D[rr * 5 + cc] += d1;
                }
            if (BS == 6) d35 += js.sa_jac[2 * int64_t(fc)];
        }
        warp_store_blocks<MT, BS>(stage, pos, inner, vals);
    }
    if (valid) {
        const double al = f.alpha[c];
#pragma unroll
        for (int rr = 0; rr < 5; ++rr)
#pragma unroll
            for (int cc = 0; cc < 5; ++cc)
                stage[lane][rr * BS + cc] = to_mt<MT>(rr == cc ? D[rr * 5 + cc] + al : D[rr * 5 + cc]);
        if (BS == 6) {
#pragma unroll
            for (int k = 0; k < 5; ++k) {
                stage[lane][k * BS + 5] = MT(0);
                stage[lane][5 * BS + k] = MT(0);
            }
            stage[lane][BS * BS - 1] = to_mt<MT>(d35 + js.sa_dsrc[c] + al);
        }
    }
    warp_store_blocks<MT, BS>(stage, js.diag[rs], valid, vals);
}

}  // namespace

template <typename MT, bool FULL>
static void launch_jacobian_t(const DevMesh& m, const DevFields& f, const GasParams& g, const JacStructure& js, int bs,
                              bool visc, MT* values, cudaStream_t s) {
    const unsigned gr = grid_for(m.n, 128);
    if (bs == 5) {
        if (visc) k_jac_rows<MT, true, 5, FULL><<<gr, 128, 0, s>>>(m, f, g, js, values);
        else k_jac_rows<MT, false, 5, FULL><<<gr, 128, 0, s>>>(m, f, g, js, values);
    } else {
        if (visc) k_jac_rows<MT, true, 6, FULL><<<gr, 128, 0, s>>>(m, f, g, js, values);
        else k_jac_rows<MT, false, 6, FULL><<<gr, 128, 0, s>>>(m, f, g, js, values);
    }
}

template <typename MT>
void launch_jacobian(const DevMesh& m, const DevFields& f, const GasParams& g, const JacStructure& js, int bs,
                     bool visc, MT* values, cudaStream_t s) {
    if (js.full_viscous && visc) launch_jacobian_t<MT, true>(m, f, g, js, bs, visc, values, s);
    else launch_jacobian_t<MT, false>(m, f, g, js, bs, visc, values, s);
}

template void launch_jacobian<double>(const DevMesh&, const DevFields&, const GasParams&, const JacStructure&, int,
                                      bool, double*, cudaStream_t);
template void launch_jacobian<float>(const DevMesh&, const DevFields&, const GasParams&, const JacStructure&, int,
                                     bool, float*, cudaStream_t);

}  // namespace cfdg
