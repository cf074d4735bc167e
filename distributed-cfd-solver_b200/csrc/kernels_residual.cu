// Residual pipeline kernels (Solver::evaluate_residual,
// include/cfd/solver/compressible/solver.hpp:169-247) and the per-cell
// time-step / right-hand-side pass (compute_dt solver.hpp:256-287,
// set_rhs_and_zero_du time/implicit_euler.hpp:81-92; du is zeroed in the linear solve).
//
// Face-to-cell accumulation is a deterministic cell-centric gather: the
// face kernel writes each face flux once, the cell kernel sums the fluxes of
// its faces in ascending face order, which is exactly the order in which the
// sequential reference scatter (residual_kernel.hpp:175-306) adds them.
#include "kernels.hpp"
#include "physics.cuh"

namespace cfdg {

namespace {

// Step 1 + 3: conserved -> primitive on cells, BC ghost primitives on
// boundary faces (the owner primitive is recomputed from U with the same
// arithmetic, so ghost and cell values agree bit for bit).
__global__ void k_primitives(DevMesh m, DevFields f, GasParams g) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t n = m.n, nt = m.nt;
    if (t < n) {
        const double U[5] = {f.U[t], f.U[n + t], f.U[2 * n + t], f.U[3 * n + t], f.U[4 * n + t]};
        double p, u, v, w, T;
        cons_to_prim(g, U, p, u, v, w, T);
        f.q[t] = p;
        f.q[nt + t] = u;
        f.q[2 * nt + t] = v;
        f.q[3 * nt + t] = w;
        f.q[4 * nt + t] = T;
    } else if (t < n + m.nb) {
        const int64_t b = t - n;
        const int32_t fc = m.ni + static_cast<int32_t>(b);
        const int32_t c0 = m.owner[fc];
        const double U[5] = {f.U[c0], f.U[n + c0], f.U[2 * n + c0], f.U[3 * n + c0], f.U[4 * n + c0]};
        double qi[5];
        cons_to_prim(g, U, qi[0], qi[1], qi[2], qi[3], qi[4]);
        const double nx = m.fnx[fc], ny = m.fny[fc], nz = m.fnz[fc];
        const double rcfn = (m.fcx[fc] - m.ccx[c0]) * nx + (m.fcy[fc] - m.ccy[c0]) * ny + (m.fcz[fc] - m.ccz[c0]) * nz;
        double qg[5];
        ghost_values(m.patches[m.bpatch[b]], g, qi, nx, ny, nz, rcfn, qg);
        for (int v = 0; v < 5; ++v) f.q[v * nt + t] = qg[v];
    }
}

// Step 5: least-squares gradient, grad(q)_c = sum_j C_j (q_j - q_c) over the
// precomputed stencil (apply_kernel_lsqf / apply_kernel_lsqn,
// src/numerics/gradient/gradient_operator.cpp:340-391,549-599).
// NVG variables starting at src (stride nt), written to dst planes.
template <int NVG>
__global__ void __launch_bounds__(128) k_gradient(DevMesh m, const double* __restrict__ src, double* __restrict__ dst) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const int32_t slice = c >> 5;
    if (int64_t(slice) * 32 >= m.n) return;  // whole warps only
    const bool act = c < m.n;
    const int lane = threadIdx.x & 31;
    const int64_t nt = m.nt;
    const int32_t cc = act ? c : m.n - 1;
    double qc[NVG], gx[NVG], gy[NVG], gz[NVG];
#pragma unroll
    for (int v = 0; v < NVG; ++v) {
        qc[v] = src[v * nt + cc];
        gx[v] = 0.0;
        gy[v] = 0.0;
        gz[v] = 0.0;
    }
    const int64_t s0 = m.g_soff[slice] + lane, s1 = m.g_soff[slice + 1];
#pragma unroll 4
    for (int64_t j = s0; j < s1; j += 32) {
        const int32_t nb = m.g_col[j];
        const double wx = m.g_wx[j], wy = m.g_wy[j], wz = m.g_wz[j];
#pragma unroll
        for (int v = 0; v < NVG; ++v) {
            const double d = src[v * nt + nb] - qc[v];
            gx[v] += wx * d;
            gy[v] += wy * d;
            gz[v] += wz * d;
        }
    }
    if (!act) return;
#pragma unroll
    for (int v = 0; v < NVG; ++v) {
        dst[(v * 3 + 0) * nt + c] = gx[v];
        dst[(v * 3 + 1) * nt + c] = gy[v];
        dst[(v * 3 + 2) * nt + c] = gz[v];
    }
}

// Step 5 (continued): ghost gradients on boundary faces
// (BoundaryManager::update_ghost_cells_grad, bc_manager.hpp:201-210) and the
// MUSCL multidimensional limiter on cells (Muscl::compute_limiters,
// numerics/reconstruction/muscl.hpp:25-105).  Threads [0,n) limiter,
// [n, n+nb) ghosts.
template <bool LIMIT, int LIM>
__global__ void __launch_bounds__(128) k_limiter_ghostgrad(DevMesh m, DevFields f, GasParams g, double k3) {
    // without the limiter (frozen or first order) the grid covers the ghosts only
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x + (LIMIT ? 0 : int64_t(m.n));
    const int64_t n = m.n, nt = m.nt;
    if (t < n) {
        if (!LIMIT) return;
        const int32_t c = static_cast<int32_t>(t);
        double qc[5], qmax[5], qmin[5], ph[5], gxc[5], gyc[5], gzc[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            qc[v] = f.q[v * nt + c];
            qmax[v] = qc[v];
            qmin[v] = qc[v];
            ph[v] = 1.0;
            gxc[v] = f.grad[(v * 3 + 0) * nt + c];
            gyc[v] = f.grad[(v * 3 + 1) * nt + c];
            gzc[v] = f.grad[(v * 3 + 2) * nt + c];
        }
        for (int32_t j = m.c2c_off[c]; j < m.c2c_off[c + 1]; ++j) {
            const int32_t nb = m.c2c[j];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                const double qn = f.q[v * nt + nb];
                qmax[v] = fmax(qmax[v], qn);
                qmin[v] = fmin(qmin[v], qn);
            }
        }
        const double eps2 = k3 * m.vol[c];
        const double cx = m.ccx[c], cy = m.ccy[c], cz = m.ccz[c];
        for (int32_t e = m.c2f_off[c]; e < m.c2f_off[c + 1]; ++e) {
            const int32_t fc = m.c2f[e];
            const double ex = m.fcx[fc] - cx, ey = m.fcy[fc] - cy, ez = m.fcz[fc] - cz;
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                const double df = gxc[v] * ex + gyc[v] * ey + gzc[v] * ez;
                const double dnb = (df > 0.0) ? (qmax[v] - qc[v]) : (qmin[v] - qc[v]);
                ph[v] = fmin(ph[v], limiter_phi<LIM>(dnb, df, eps2));
            }
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) f.phi[v * n + c] = ph[v];
    } else if (t < n + m.nb) {
        const int64_t b = t - n;
        const int32_t fc = m.ni + static_cast<int32_t>(b);
        const int32_t c0 = m.owner[fc];
        const double nx = m.fnx[fc], ny = m.fny[fc], nz = m.fnz[fc];
        const double rcfn = (m.fcx[fc] - m.ccx[c0]) * nx + (m.fcy[fc] - m.ccy[c0]) * ny + (m.fcz[fc] - m.ccz[c0]) * nz;
        const double rcfn_inv = 1.0 / fmax(rcfn, 1.0e-14);
        double gi[5][3], gg[5][3], qi[5], qgh[5];
        for (int v = 0; v < 5; ++v) {
            qi[v] = f.q[v * nt + c0];
            qgh[v] = f.q[v * nt + t];
            for (int d = 0; d < 3; ++d) gi[v][d] = f.grad[(v * 3 + d) * nt + c0];
        }
        ghost_gradients(m.patches[m.bpatch[b]], g, gi, qi, qgh, nx, ny, nz, rcfn_inv, gg);
        for (int v = 0; v < 5; ++v)
            for (int d = 0; d < 3; ++d) f.grad[(v * 3 + d) * nt + t] = gg[v][d];
    }
}

// Step 6: one thread per face evaluates MUSCL states (interior faces) or
// first-order states (boundary faces), HLLC, and the viscous flux
// (ResidualKernel::compute_fluxes, residual_kernel.hpp:175-306), and stores
// F (5) and A*s_max (+ viscous radius) for the cell gather.
template <bool MUSCL, bool VISC>
__global__ void __launch_bounds__(128, VISC ? 0 : 6) k_face_flux(DevMesh m, DevFields f, GasParams g) {
    const int32_t fc = blockIdx.x * blockDim.x + threadIdx.x;
    if (fc >= m.nf) return;
    const int64_t nt = m.nt;
    const bool inner = fc < m.ni;
    const int32_t c0 = m.owner[fc];
    const int32_t c1 = inner ? m.neigh[fc] : m.n + (fc - m.ni);
    const double nx = m.fnx[fc], ny = m.fny[fc], nz = m.fnz[fc], A = m.farea[fc];
    double qL[5], qR[5];
    if (MUSCL && inner) {
        const double fx = m.fcx[fc], fy = m.fcy[fc], fz = m.fcz[fc];
        const double d0x = fx - m.ccx[c0], d0y = fy - m.ccy[c0], d0z = fz - m.ccz[c0];
        const double d1x = fx - m.ccx[c1], d1y = fy - m.ccy[c1], d1z = fz - m.ccz[c1];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const double dot0 = f.grad[(v * 3 + 0) * nt + c0] * d0x + f.grad[(v * 3 + 1) * nt + c0] * d0y +
                                f.grad[(v * 3 + 2) * nt + c0] * d0z;
            qL[v] = f.q[v * nt + c0] + f.phi[v * m.n + c0] * dot0;
            const double dot1 = f.grad[(v * 3 + 0) * nt + c1] * d1x + f.grad[(v * 3 + 1) * nt + c1] * d1y +
                                f.grad[(v * 3 + 2) * nt + c1] * d1z;
            qR[v] = f.q[v * nt + c1] + f.phi[v * m.n + c1] * dot1;
        }
    } else {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            qL[v] = f.q[v * nt + c0];
            qR[v] = f.q[v * nt + c1];
        }
    }
    double UL[5], UR[5], F[5], smax;
    prim_to_cons(g, qL[0], qL[1], qL[2], qL[3], qL[4], UL);
    prim_to_cons(g, qR[0], qR[1], qR[2], qR[3], qR[4], UR);
    hllc_flux(g, UL, UR, nx, ny, nz, A, F, smax);
    double lam_f = A * smax;
    if (VISC) {
        double qcL[5], qcR[5], gL[12], gR[12];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            qcL[v] = f.q[v * nt + c0];
            qcR[v] = f.q[v * nt + c1];
        }
#pragma unroll
        for (int v = 1; v < 5; ++v)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                gL[(v - 1) * 3 + d] = f.grad[(v * 3 + d) * nt + c0];
                gR[(v - 1) * 3 + d] = f.grad[(v * 3 + d) * nt + c1];
            }
        const double mutL = f.mut ? f.mut[c0] : 0.0;
        const double mutR = f.mut ? f.mut[c1] : 0.0;
        const ViscGeom geo{m.finv_d[fc], m.fdx[fc], m.fdy[fc], m.fdz[fc]};
        double Fv[5];
        const double lv = viscous_flux(g, geo, qcL, qcR, gL, gR, mutL, mutR, nx, ny, nz, A, Fv);
#pragma unroll
        for (int v = 1; v < 5; ++v) F[v] += Fv[v];
        lam_f += lv;
    }
    // face-major: the face's 5 fluxes and A*s_max are one 48-byte record
    double2* dst = reinterpret_cast<double2*>(f.fflux + int64_t(fc) * 6);
    dst[0] = make_double2(F[0], F[1]);
    dst[1] = make_double2(F[2], F[3]);
    dst[2] = make_double2(F[4], lam_f);
}

// Cell gather of face fluxes into R and lam (ascending face order).
__global__ void __launch_bounds__(256) k_cell_residual(DevMesh m, DevFields f) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.n) return;
    const int64_t n = m.n;
    double r[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    double l = 0.0;
    for (int32_t e = m.c2f_off[c]; e < m.c2f_off[c + 1]; ++e) {
        const int32_t es = __ldg(m.c2fs + e);  // the side is in the sign: no owner gather
        const int32_t fc = es >= 0 ? es : ~es;
        const double2* rec = reinterpret_cast<const double2*>(f.fflux + int64_t(fc) * 6);
        const double2 a = __ldg(rec), b = __ldg(rec + 1), d = __ldg(rec + 2);
        const double F[5] = {a.x, a.y, b.x, b.y, d.x};
        if (es >= 0) {
#pragma unroll
            for (int v = 0; v < 5; ++v) r[v] += F[v];
        } else {
#pragma unroll
            for (int v = 0; v < 5; ++v) r[v] -= F[v];
        }
        l += d.y;
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) f.res[v * n + c] = r[v];
    f.lam[c] = l;
}

// Per-block partial sums of R_v^2 over cells (Solver::residual_norms,
// solver.hpp:740-756); summed in fixed order by finalize_norms.
template <int NV>
__global__ void __launch_bounds__(256) k_norm_partials(int32_t n, const double* __restrict__ res, double* __restrict__ partials) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    double sq[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const double r = (c < n) ? res[int64_t(v) * n + c] : 0.0;
        sq[v] = r * r;
    }
    block_reduce_store<NV, 256>(sq, partials + size_t(blockIdx.x) * NV);
}

// Warp v sums column v of the partials (lane-strided, then a fixed shuffle
// tree): deterministic for a given block count.
__global__ void k_norm_finalize(int nblocks, int nv, const double* __restrict__ partials, double scale,
                                double* __restrict__ l2) {
    const int v = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (v >= nv) return;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += partials[size_t(b) * nv + v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) l2[v] = sqrt(s * scale);
}

// compute_dt (solver.hpp:263-277) fused with the right-hand side of
// set_rhs_and_zero_du (implicit_euler.hpp:81-92): alpha = max(lam,floor)/CFL,
// b = -R (AoS).  The update du starts from zero (or the learned guess) in
// the linear solve itself.  A 6-variable row of b is 48 bytes and stores as
// three 16-byte pairs.
template <int NV>
__global__ void k_dt_rhs(DevMesh m, DevFields f, double cfl, double diag, double* __restrict__ b) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.n) return;
    const int64_t n = m.n;
    const double inv_cfl = 1.0 / cfl;
    const double l = fmax(f.lam[c], kLamFloor);
    f.dt[c] = cfl * m.vol[c] / l;
    f.alpha[c] = (l * inv_cfl) + (m.vol[c] * diag);  // diag: BDF coefficient / dt (0 when steady)
    if (b) {
        const int64_t r = row_index(m, c);
        double v6[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) v6[v] = -f.res[v * n + c];
        if constexpr (NV == 6) {
            double2* dst = reinterpret_cast<double2*>(b + r * NV);
#pragma unroll
            for (int h = 0; h < 3; ++h) dst[h] = make_double2(v6[2 * h], v6[2 * h + 1]);
        } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) b[r * NV + v] = v6[v];
        }
    }
}

// U <- U + du (AoS du), implicit_euler.hpp:49-61; SA variable clamped at 0
// (SpalartAllmaras::post_stage).  `scale` (device scalar, may be null):
// U <- U + scale * du, the relaxed Jacobian-free step.
template <int NV>
__global__ void k_state_update(DevMesh m, double* __restrict__ U, const double* __restrict__ du,
                               const double* __restrict__ scale) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.n) return;
    const int64_t n = m.n;
    const int64_t r = row_index(m, c);
    const double w = scale ? *scale : 1.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        double x = scale ? U[v * n + c] + w * du[r * NV + v] : U[v * n + c] + du[r * NV + v];
        if (v == 5 && x < 0.0) x = 0.0;
        U[v * n + c] = x;
    }
}

__global__ void k_fill(double* __restrict__ x, int64_t count, double value) {
    const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) x[i] = value;
}

}  // namespace

void launch_primitives(const DevMesh& m, const DevFields& f, const GasParams& g, cudaStream_t s) {
    const int64_t th = int64_t(m.n) + m.nb;
    k_primitives<<<grid_for(th, 256), 256, 0, s>>>(m, f, g);
}

void launch_gradient(const DevMesh& m, const double* src, double* dst, int nvars, cudaStream_t s) {
    const unsigned gr = grid_for(m.n, 128);
    switch (nvars) {
        case 1: k_gradient<1><<<gr, 128, 0, s>>>(m, src, dst); break;
        case 5: k_gradient<5><<<gr, 128, 0, s>>>(m, src, dst); break;
        case 6: k_gradient<6><<<gr, 128, 0, s>>>(m, src, dst); break;  // 5 primitives + nu_tilde
        default: break;
    }
}

void launch_limiter_ghostgrad(const DevMesh& m, const DevFields& f, const GasParams& g, bool limit, int limiter,
                              double venkat_k, cudaStream_t s) {
    const double k3 = venkat_k * venkat_k * venkat_k;
    const int64_t th = int64_t(m.n) + m.nb;
    const unsigned gr = grid_for(th, 128);
    if (!limit) {
        if (m.nb > 0) k_limiter_ghostgrad<false, 1><<<grid_for(m.nb, 128), 128, 0, s>>>(m, f, g, k3);
    } else if (limiter == 2) {
        k_limiter_ghostgrad<true, 2><<<gr, 128, 0, s>>>(m, f, g, k3);
    } else if (limiter == 3) {
        k_limiter_ghostgrad<true, 3><<<gr, 128, 0, s>>>(m, f, g, k3);
    } else {
        k_limiter_ghostgrad<true, 1><<<gr, 128, 0, s>>>(m, f, g, k3);
    }
}

void launch_face_flux(const DevMesh& m, const DevFields& f, const GasParams& g, bool muscl, bool visc,
                      cudaStream_t s) {
    const unsigned gr = grid_for(m.nf, 128);
    if (muscl && visc) k_face_flux<true, true><<<gr, 128, 0, s>>>(m, f, g);
    else if (muscl) k_face_flux<true, false><<<gr, 128, 0, s>>>(m, f, g);
    else if (visc) k_face_flux<false, true><<<gr, 128, 0, s>>>(m, f, g);
    else k_face_flux<false, false><<<gr, 128, 0, s>>>(m, f, g);
}

void launch_cell_residual(const DevMesh& m, const DevFields& f, cudaStream_t s) {
    k_cell_residual<<<grid_for(m.n, 256), 256, 0, s>>>(m, f);
}

int norm_blocks(int32_t n) { return static_cast<int>(grid_for(n, 256)); }

void launch_norms(int32_t n, int nv, const double* res, double* partials, double* l2, cudaStream_t s) {
    const unsigned gr = grid_for(n, 256);
    if (nv == 6) k_norm_partials<6><<<gr, 256, 0, s>>>(n, res, partials);
    else k_norm_partials<5><<<gr, 256, 0, s>>>(n, res, partials);
    k_norm_finalize<<<1, 32 * 6, 0, s>>>(static_cast<int>(gr), nv, partials, 1.0 / double(n > 0 ? n : 1), l2);
}

void launch_dt_rhs(const DevMesh& m, const DevFields& f, int nv, double cfl, double diag, double* b, cudaStream_t s) {
    const unsigned gr = grid_for(m.n, 256);
    if (nv == 6) k_dt_rhs<6><<<gr, 256, 0, s>>>(m, f, cfl, diag, b);
    else k_dt_rhs<5><<<gr, 256, 0, s>>>(m, f, cfl, diag, b);
}

// Dual-time pseudo-source (Solver::add_unsteady_source_term,
// solver.hpp:546-580): res += V (c0 U + c1 U^n + c2 U^{n-1}); BDF1 has c2 = 0
// and reads no U^{n-1}.
__global__ void k_unsteady_source(int32_t n, int nv, const double* __restrict__ vol, const double* __restrict__ U,
                                  const double* __restrict__ Un, const double* __restrict__ Unm1, double c0,
                                  double c1, double c2, double* __restrict__ res) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= int64_t(n) * nv) return;
    const int32_t c = static_cast<int32_t>(t % n);
    const double src = Unm1 ? (c0 * U[t] + c1 * Un[t] + c2 * Unm1[t]) : (c0 * U[t] + c1 * Un[t]);
    res[t] += vol[c] * src;
}

void launch_unsteady_source(int32_t n, int nv, const double* vol, const double* U, const double* Un,
                            const double* Unm1, double c0, double c1, double c2, double* res, cudaStream_t s) {
    const int64_t len = int64_t(n) * nv;
    if (len > 0) k_unsteady_source<<<grid_for(len, 256), 256, 0, s>>>(n, nv, vol, U, Un, Unm1, c0, c1, c2, res);
}

void launch_state_update(const DevMesh& m, double* U, const double* du, int nv, const double* scale, cudaStream_t s) {
    const unsigned gr = grid_for(m.n, 256);
    if (nv == 6) k_state_update<6><<<gr, 256, 0, s>>>(m, U, du, scale);
    else k_state_update<5><<<gr, 256, 0, s>>>(m, U, du, scale);
}

void launch_fill(double* x, int64_t count, double value, cudaStream_t s) {
    if (count <= 0) return;
    k_fill<<<grid_for(count, 256), 256, 0, s>>>(x, count, value);
}

}  // namespace cfdg
