// Gradient and limiter kernels over caller-owned per-variable arrays
// (cfdg_gradient / cfdg_limiter).  The arithmetic is that of the solver's
// own kernels (k_gradient, k_limiter_ghostgrad in kernels_residual.cu); only
// the field addressing differs: one pointer per variable instead of planes
// of one allocation.
#include "physics.cuh"
#include "recon.hpp"

namespace cfdg {
namespace {

// grad(q)_c = sum_j C_j (q_j - q_c) over the warp-sliced stencil
// (apply_kernel_lsqf / apply_kernel_lsqn,
// src/numerics/gradient/gradient_operator.cpp:340-391,549-599).
template <int NV>
__global__ void __launch_bounds__(128) k_gradient_ptrs(DevMesh m, ReconPtrs p) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    const int32_t slice = c >> 5;
    if (int64_t(slice) * 32 >= m.n) return;  // whole warps only
    const bool act = c < m.n;
    const int lane = threadIdx.x & 31;
    const int32_t cc = act ? c : m.n - 1;
    double qc[NV], gx[NV], gy[NV], gz[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        qc[v] = p.q[v][cc];
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
        for (int v = 0; v < NV; ++v) {
            const double d = p.q[v][nb] - qc[v];
            gx[v] += wx * d;
            gy[v] += wy * d;
            gz[v] += wz * d;
        }
    }
    if (!act) return;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        p.out[3 * v + 0][c] = gx[v];
        p.out[3 * v + 1][c] = gy[v];
        p.out[3 * v + 2][c] = gz[v];
    }
}

// Neighbour extrema over the face neighbours, then the minimum over the
// cell's faces of the limiter function (Muscl::compute_limiters,
// numerics/reconstruction/muscl.hpp:25-105).
template <int NV, int LIM>
__global__ void __launch_bounds__(128) k_limiter_ptrs(DevMesh m, ReconPtrs p, double k3) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.n) return;
    double qc[NV], qmax[NV], qmin[NV], ph[NV], gxc[NV], gyc[NV], gzc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        qc[v] = p.q[v][c];
        qmax[v] = qc[v];
        qmin[v] = qc[v];
        ph[v] = 1.0;
        gxc[v] = p.gx[v][c];
        gyc[v] = p.gy[v][c];
        gzc[v] = p.gz[v][c];
    }
    for (int32_t j = m.c2c_off[c]; j < m.c2c_off[c + 1]; ++j) {
        const int32_t nb = m.c2c[j];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            const double qn = p.q[v][nb];
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
        for (int v = 0; v < NV; ++v) {
            const double df = gxc[v] * ex + gyc[v] * ey + gzc[v] * ez;
            const double dnb = (df > 0.0) ? (qmax[v] - qc[v]) : (qmin[v] - qc[v]);
            ph[v] = fmin(ph[v], limiter_phi<LIM>(dnb, df, eps2));
        }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) p.out[v][c] = ph[v];
}

}  // namespace

template <int NV>
void launch_gradient_ptrs(const DevMesh& m, const ReconPtrs& p, cudaStream_t s) {
    const int64_t threads = (int64_t(m.n) + 31) / 32 * 32;
    k_gradient_ptrs<NV><<<grid_for(threads, 128), 128, 0, s>>>(m, p);
}

template <int NV>
void launch_limiter_ptrs(const DevMesh& m, const ReconPtrs& p, int limiter, double k3, cudaStream_t s) {
    const unsigned grid = grid_for(m.n, 128);
    if (limiter == CFDG_LIM_BARTH_JESPERSEN) k_limiter_ptrs<NV, CFDG_LIM_BARTH_JESPERSEN><<<grid, 128, 0, s>>>(m, p, k3);
    else if (limiter == CFDG_LIM_VAN_ALBADA) k_limiter_ptrs<NV, CFDG_LIM_VAN_ALBADA><<<grid, 128, 0, s>>>(m, p, k3);
    else k_limiter_ptrs<NV, CFDG_LIM_VENKATAKRISHNAN><<<grid, 128, 0, s>>>(m, p, k3);
}

#define CFDG_RECON_INST(NV)                                                                   \
    template void launch_gradient_ptrs<NV>(const DevMesh&, const ReconPtrs&, cudaStream_t);  \
    template void launch_limiter_ptrs<NV>(const DevMesh&, const ReconPtrs&, int, double, cudaStream_t);
CFDG_RECON_INST(1)
CFDG_RECON_INST(2)
CFDG_RECON_INST(3)
CFDG_RECON_INST(4)
CFDG_RECON_INST(5)
CFDG_RECON_INST(6)
#undef CFDG_RECON_INST

// ------------------------------------------------------------ the operator
ReconOperator::ReconOperator(int device, const cfdg_mesh_host& mesh, int gradient, int limiter, double venkat_k)
    : device_(device), limiter_(limiter), k3_(venkat_k * venkat_k * venkat_k) {
    if (gradient != CFDG_GRAD_LSQ_FACE && gradient != CFDG_GRAD_LSQ_NODE)
        throw Failure{CFDG_ERR_UNSUPPORTED, "gradient operator not built (least-squares face or node only)"};
    if (limiter != CFDG_LIM_VENKATAKRISHNAN && limiter != CFDG_LIM_BARTH_JESPERSEN && limiter != CFDG_LIM_VAN_ALBADA)
        throw Failure{CFDG_ERR_INVALID, "unknown limiter"};
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    HostMesh hm;
    hm.from_view(mesh);
    const cudaStream_t s = nullptr;
    dm_.n = hm.n_cells;
    dm_.nf = hm.n_faces;
    dm_.ni = hm.n_inner;
    dm_.nb = hm.n_faces - hm.n_inner;
    dm_.nt = dm_.n + dm_.nb;
    const Csr c2f = build_cell_faces(hm);
    const Csr c2c = build_cell_cells_face(hm);
    const LsqSlices sl = build_lsq_slices(hm, gradient == CFDG_GRAD_LSQ_FACE ? c2c : build_cell_cells_node(hm));
    upload_or_throw(c2f_off_, c2f.off, s, "c2f_off");
    upload_or_throw(c2f_, c2f.val, s, "c2f");
    upload_or_throw(c2c_off_, c2c.off, s, "c2c_off");
    upload_or_throw(c2c_, c2c.val, s, "c2c");
    upload_or_throw(g_soff_, sl.soff, s, "g_soff");
    upload_or_throw(g_col_, sl.col, s, "g_col");
    upload_or_throw(g_wx_, sl.wx, s, "g_wx");
    upload_or_throw(g_wy_, sl.wy, s, "g_wy");
    upload_or_throw(g_wz_, sl.wz, s, "g_wz");
    upload_or_throw(fcx_, hm.fcx, s, "fcx");
    upload_or_throw(fcy_, hm.fcy, s, "fcy");
    upload_or_throw(fcz_, hm.fcz, s, "fcz");
    upload_or_throw(ccx_, hm.ccx, s, "ccx");
    upload_or_throw(ccy_, hm.ccy, s, "ccy");
    upload_or_throw(ccz_, hm.ccz, s, "ccz");
    upload_or_throw(vol_, hm.vol, s, "vol");
    cuda_check(cudaStreamSynchronize(s), "setup sync");  // the host vectors die at scope end
    dm_.c2f_off = c2f_off_.p;
    dm_.c2f = c2f_.p;
    dm_.c2c_off = c2c_off_.p;
    dm_.c2c = c2c_.p;
    dm_.g_soff = g_soff_.p;
    dm_.g_col = g_col_.p;
    dm_.g_wx = g_wx_.p;
    dm_.g_wy = g_wy_.p;
    dm_.g_wz = g_wz_.p;
    dm_.fcx = fcx_.p;
    dm_.fcy = fcy_.p;
    dm_.fcz = fcz_.p;
    dm_.ccx = ccx_.p;
    dm_.ccy = ccy_.p;
    dm_.ccz = ccz_.p;
    dm_.vol = vol_.p;
}

namespace {
template <typename F>
void by_chunks(int nvars, F&& f) {
    for (int v0 = 0; v0 < nvars; v0 += kMaxVars) f(v0, std::min(kMaxVars, nvars - v0));
}
template <typename L>
void dispatch_nv(int nv, L&& launch) {
    switch (nv) {
        case 1: launch(std::integral_constant<int, 1>{}); break;
        case 2: launch(std::integral_constant<int, 2>{}); break;
        case 3: launch(std::integral_constant<int, 3>{}); break;
        case 4: launch(std::integral_constant<int, 4>{}); break;
        case 5: launch(std::integral_constant<int, 5>{}); break;
        default: launch(std::integral_constant<int, 6>{}); break;
    }
}
}  // namespace

void ReconOperator::gradient(const double* const* q, double* const* gx, double* const* gy, double* const* gz,
                             int nvars, cudaStream_t s) {
    if (nvars < 1 || !q || !gx || !gy || !gz) throw Failure{CFDG_ERR_INVALID, "cfdg_gradient: empty field set"};
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    by_chunks(nvars, [&](int v0, int nv) {
        ReconPtrs p{};
        for (int v = 0; v < nv; ++v) {
            if (!q[v0 + v] || !gx[v0 + v] || !gy[v0 + v] || !gz[v0 + v])
                throw Failure{CFDG_ERR_INVALID, "cfdg_gradient: null field pointer"};
            p.q[v] = q[v0 + v];
            p.out[3 * v] = gx[v0 + v];
            p.out[3 * v + 1] = gy[v0 + v];
            p.out[3 * v + 2] = gz[v0 + v];
        }
        if (dm_.n > 0) dispatch_nv(nv, [&](auto k) { launch_gradient_ptrs<decltype(k)::value>(dm_, p, s); });
    });
    cuda_check(cudaGetLastError(), "gradient launch");
}

void ReconOperator::limiter(const double* const* q, const double* const* gx, const double* const* gy,
                            const double* const* gz, double* const* phi, int nvars, cudaStream_t s) {
    if (nvars < 1 || !q || !gx || !gy || !gz || !phi) throw Failure{CFDG_ERR_INVALID, "cfdg_limiter: empty field set"};
    cuda_check(cudaSetDevice(device_), "cudaSetDevice");
    by_chunks(nvars, [&](int v0, int nv) {
        ReconPtrs p{};
        for (int v = 0; v < nv; ++v) {
            if (!q[v0 + v] || !gx[v0 + v] || !gy[v0 + v] || !gz[v0 + v] || !phi[v0 + v])
                throw Failure{CFDG_ERR_INVALID, "cfdg_limiter: null field pointer"};
            p.q[v] = q[v0 + v];
            p.gx[v] = gx[v0 + v];
            p.gy[v] = gy[v0 + v];
            p.gz[v] = gz[v0 + v];
            p.out[v] = phi[v0 + v];
        }
        if (dm_.n > 0)
            dispatch_nv(nv, [&](auto k) { launch_limiter_ptrs<decltype(k)::value>(dm_, p, limiter_, k3_, s); });
    });
    cuda_check(cudaGetLastError(), "limiter launch");
}

}  // namespace cfdg
