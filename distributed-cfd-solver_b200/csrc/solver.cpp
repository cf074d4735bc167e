// Host orchestration of the GPU hot path: set-up (connectivity, LSQ
// coefficients, BSR structure, SGS orderings, boundary table), the residual
// pipeline, Jacobian assembly, BiCGSTAB + SGS and the Newton loop.
#include "solver.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <queue>

namespace cfdg {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        throw Failure{e == cudaErrorMemoryAllocation ? CFDG_ERR_NOMEM : CFDG_ERR_CUDA,
                      std::string(what) + ": " + cudaGetErrorString(e)};
    }
}

namespace {

// invert3x3 of the least-squares setup (gradient_operator.cpp:20-47).
bool invert3x3(const double A[9], double inv[9]) {
    const double eps = 1.0e-14;
    const double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
                       A[2] * (A[3] * A[7] - A[4] * A[6]);
    if (std::abs(det) <= eps) {
        std::fill_n(inv, 9, 0.0);
        return false;
    }
    const double id = 1.0 / det;
    inv[0] = (A[4] * A[8] - A[5] * A[7]) * id;
    inv[1] = (A[2] * A[7] - A[1] * A[8]) * id;
    inv[2] = (A[1] * A[5] - A[2] * A[4]) * id;
    inv[3] = (A[5] * A[6] - A[3] * A[8]) * id;
    inv[4] = (A[0] * A[8] - A[2] * A[6]) * id;
    inv[5] = (A[2] * A[3] - A[0] * A[5]) * id;
    inv[6] = (A[3] * A[7] - A[4] * A[6]) * id;
    inv[7] = (A[1] * A[6] - A[0] * A[7]) * id;
    inv[8] = (A[0] * A[4] - A[1] * A[3]) * id;
    return true;
}

// Weighted least-squares coefficients C_j = A^-1 w_j dr_j, w = 1/|dr|^2,
// A = sum w dr dr^T + 1e-14 I (LeastSquaresCell{Face,Node}Gradient::setup,
// gradient_operator.cpp:414-499, 622-707).
void lsq_coefficients(const HostMesh& m, const Csr& st, std::vector<double>& wx, std::vector<double>& wy,
                      std::vector<double>& wz) {
    wx.assign(st.val.size(), 0.0);
    wy.assign(st.val.size(), 0.0);
    wz.assign(st.val.size(), 0.0);
    std::vector<double> dr, w;
    for (int32_t c = 0; c < m.n_cells; ++c) {
        const int32_t p1 = st.off[c], p2 = st.off[c + 1];
        const int32_t nn = p2 - p1;
        if (nn == 0) continue;
        const double x0 = m.ccx[c], y0 = m.ccy[c], z0 = m.ccz[c];
        dr.resize(3 * static_cast<std::size_t>(nn));
        w.resize(nn);
        double A[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int32_t i = 0; i < nn; ++i) {
            const int32_t nb = st.val[p1 + i];
            const double dx = m.ccx[nb] - x0, dy = m.ccy[nb] - y0, dz = m.ccz[nb] - z0;
            const double r2 = dx * dx + dy * dy + dz * dz;
            const double ww = 1.0 / std::max(r2, 1.0e-30);
            dr[3 * i] = dx;
            dr[3 * i + 1] = dy;
            dr[3 * i + 2] = dz;
            w[i] = ww;
            A[0] += ww * dx * dx;
            A[1] += ww * dx * dy;
            A[2] += ww * dx * dz;
            A[4] += ww * dy * dy;
            A[5] += ww * dy * dz;
            A[8] += ww * dz * dz;
        }
        A[3] = A[1];
        A[6] = A[2];
        A[7] = A[5];
        A[0] += 1.0e-14;
        A[4] += 1.0e-14;
        A[8] += 1.0e-14;
        double inv[9];
        invert3x3(A, inv);
        for (int32_t i = 0; i < nn; ++i) {
            const double rx = w[i] * dr[3 * i], ry = w[i] * dr[3 * i + 1], rz = w[i] * dr[3 * i + 2];
            wx[p1 + i] = inv[0] * rx + inv[1] * ry + inv[2] * rz;
            wy[p1 + i] = inv[3] * rx + inv[4] * ry + inv[5] * rz;
            wz[p1 + i] = inv[6] * rx + inv[7] * ry + inv[8] * rz;
        }
    }
}

}  // namespace

// LSQ coefficients of the stencil `st` laid out in warp slices (see
// DevMesh::g_soff).
LsqSlices build_lsq_slices(const HostMesh& hm, const Csr& st) {
    std::vector<double> wx, wy, wz;
    lsq_coefficients(hm, st, wx, wy, wz);
    LsqSlices out;
    const int32_t n = hm.n_cells;
    const int32_t ns = (n + 31) / 32;
    out.soff.assign(static_cast<std::size_t>(ns) + 1, 0);
    for (int32_t sl = 0; sl < ns; ++sl) {
        int32_t len = 0;
        for (int32_t c = sl * 32; c < std::min(n, sl * 32 + 32); ++c) len = std::max(len, st.off[c + 1] - st.off[c]);
        out.soff[sl + 1] = out.soff[sl] + int64_t(len) * 32;
    }
    const std::size_t slots = static_cast<std::size_t>(out.soff[ns]);
    out.col.assign(slots, 0);
    out.wx.assign(slots, 0.0);
    out.wy.assign(slots, 0.0);
    out.wz.assign(slots, 0.0);
    for (int32_t sl = 0; sl < ns; ++sl) {
        const int32_t len = static_cast<int32_t>((out.soff[sl + 1] - out.soff[sl]) / 32);
        for (int l = 0; l < 32; ++l) {
            const int32_t c = sl * 32 + l;
            const int32_t cc = c < n ? c : n - 1;  // lanes past the last cell read a real cell
            for (int32_t k = 0; k < len; ++k) {
                const std::size_t q = static_cast<std::size_t>(out.soff[sl] + int64_t(k) * 32 + l);
                const int32_t j = (c < n) ? st.off[c] + k : -1;
                if (j >= 0 && j < st.off[c + 1]) {
                    out.col[q] = st.val[j];
                    out.wx[q] = wx[j];
                    out.wy[q] = wy[j];
                    out.wz[q] = wz[j];
                } else {
                    out.col[q] = cc;  // padding: own cell, zero weights
                }
            }
        }
    }
    out.entries = static_cast<int64_t>(st.val.size());
    return out;
}

namespace {

struct Inflow {
    double p, u, v, w, T;
};

// resolve_inflow of the BC registry (bc_manager.hpp:37-121).
Inflow resolve_inflow(const cfdg_bc_desc& d, const GasParams& g, double p_ref) {
    if (d.inflow_mode == CFDG_INFLOW_MACH_ANGLES) {
        const double k = M_PI / 180.0;
        const double a_r = d.alpha_deg * k, b_r = d.beta_deg * k;
        const double rho = p_ref / (g.R * d.t);
        const double a = std::sqrt(g.gamma * p_ref / rho);
        const double vm = d.mach * a;
        return {p_ref, vm * std::cos(a_r) * std::cos(b_r), -vm * std::sin(b_r), vm * std::sin(a_r) * std::cos(b_r),
                d.t};
    }
    if (d.inflow_mode == CFDG_INFLOW_MACH_DIRECTION) {
        const double rho = p_ref / (g.R * d.t);
        const double a = std::sqrt(g.gamma * p_ref / rho);
        const double vm = d.mach * a;
        const double nrm =
            std::sqrt(d.direction[0] * d.direction[0] + d.direction[1] * d.direction[1] + d.direction[2] * d.direction[2]);
        const double inv = (nrm > 1.0e-14) ? (1.0 / nrm) : 0.0;
        return {p_ref, vm * d.direction[0] * inv, vm * d.direction[1] * inv, vm * d.direction[2] * inv, d.t};
    }
    return {p_ref, d.velocity[0], d.velocity[1], d.velocity[2], d.t};
}

}  // namespace

// =============================================================== Profiler
Profiler::~Profiler() {
    for (cudaEvent_t e : all_) cudaEventDestroy(e);
}

cudaEvent_t Profiler::get() {
    if (free_.empty()) {
        cudaEvent_t e;
        cuda_check(cudaEventCreate(&e), "cudaEventCreate");
        all_.push_back(e);
        return e;
    }
    cudaEvent_t e = free_.back();
    free_.pop_back();
    return e;
}

void Profiler::enable(bool on) {
    on_ = on;
    for (int c = 0; c < CFDG_KCAT_COUNT; ++c) {
        ms[c] = 0.0;
        count[c] = 0;
        bytes[c] = 0.0;
    }
    for (const Rec& r : pending_) {
        free_.push_back(r.a);
        free_.push_back(r.b);
    }
    pending_.clear();
}

void Profiler::start(int cat, cudaStream_t s) {
    open_ = get();
    open_cat_ = cat;
    cuda_check(cudaEventRecord(open_, s), "cudaEventRecord");
}

void Profiler::stop(cudaStream_t s) {
    cudaEvent_t b = get();
    cuda_check(cudaEventRecord(b, s), "cudaEventRecord");
    pending_.push_back({open_cat_, open_, b});
    open_ = nullptr;
}

void Profiler::collect() {
    for (const Rec& r : pending_) {
        float t = 0.0f;
        cuda_check(cudaEventSynchronize(r.b), "cudaEventSynchronize");
        cuda_check(cudaEventElapsedTime(&t, r.a, r.b), "cudaEventElapsedTime");
        ms[r.cat] += t;
        count[r.cat] += 1;
        free_.push_back(r.a);
        free_.push_back(r.b);
    }
    pending_.clear();
}

// =============================================================== BsrSystem
BsrSystem::BsrSystem(int device, int32_t n, int32_t bs, const int32_t* row_ptr, const int32_t* cols, int precision,
                     cudaStream_t stream)
    : device_(device), stream_(stream), n_(n), bs_(bs), precision_(precision) {
    if (n < 0 || bs < 1 || bs > 6 || bs == 2) throw Failure{CFDG_ERR_INVALID, "unsupported BSR size or block size"};
    row_ptr_h_.assign(row_ptr, row_ptr + n + 1);
    nnzb_ = row_ptr_h_[n];
    cols_h_.assign(cols, cols + nnzb_);
    diag_h_.assign(n, -1);
    for (int32_t i = 0; i < n; ++i) {
        if (row_ptr_h_[i + 1] < row_ptr_h_[i]) throw Failure{CFDG_ERR_INVALID, "row pointers must not decrease"};
        for (int32_t k = row_ptr_h_[i]; k < row_ptr_h_[i + 1]; ++k) {
            if (cols_h_[k] < 0 || cols_h_[k] >= n) throw Failure{CFDG_ERR_INVALID, "column index out of range"};
            if (k > row_ptr_h_[i] && cols_h_[k] <= cols_h_[k - 1])
                throw Failure{CFDG_ERR_INVALID, "columns must be sorted and unique within a row"};
            if (cols_h_[k] == i) diag_h_[i] = k;
        }
        if (diag_h_[i] < 0) throw Failure{CFDG_ERR_INVALID, "block row without a diagonal block"};
    }
    upload_or_throw(row_ptr_, row_ptr_h_, stream_, "row_ptr");
    upload_or_throw(cols_, cols_h_, stream_, "cols");
    upload_or_throw(diag_, diag_h_, stream_, "diag");
    const std::size_t nv = static_cast<std::size_t>(nnzb_) * bs * bs;
    if (precision_ == CFDG_PREC_MIXED) alloc_or_throw(vals32_, nv, "values");
    else alloc_or_throw(vals64_, nv, "values");
    const std::size_t N = static_cast<std::size_t>(n) * bs;
    for (DevArray<double>* a : {&r_, &r0_, &p_, &v_, &s_, &t_, &phat_, &shat_}) alloc_or_throw(*a, N > 0 ? N : 1, "krylov");
    // the fused colour-0 product and the SpMV of the other rows write their
    // partials one after the other
    alloc_or_throw(partials_,
                   static_cast<std::size_t>(sgs_last_spmv_blocks(n, bs) + std::max(dot_blocks(N), spmv_blocks(n, bs))) * 5 + 8,
                   "partials");
    alloc_or_throw(ks_, 1, "krylov scalars");
    alloc_or_throw(err_, 1, "error flag");
    cuda_check(cudaMallocHost(reinterpret_cast<void**>(&ks_host_), sizeof(KrylovScalars)), "cudaMallocHost");
}

BsrSystem::~BsrSystem() {
    release_device_loop();
    if (ks_host_) cudaFreeHost(ks_host_);
    if (gm_h_host_) cudaFreeHost(gm_h_host_);
}

void BsrSystem::set_precision(int precision) {
    if (precision != CFDG_PREC_FP64 && precision != CFDG_PREC_MIXED) throw Failure{CFDG_ERR_INVALID, "unknown precision"};
    if (precision == precision_) return;
    const std::size_t nv = static_cast<std::size_t>(nnzb_) * bs_ * bs_;
    release_device_loop();  // the captured iteration launches precision-specific kernels
    if (precision == CFDG_PREC_MIXED) {
        vals64_.release();
        lu64_.release();
        alloc_or_throw(vals32_, nv, "values");
    } else {
        vals32_.release();
        lu32_.release();
        alloc_or_throw(vals64_, nv, "values");
    }
    precision_ = precision;
    lu_ready_ = false;
}

void BsrSystem::set_values_host(const double* v) {
    const std::size_t nv = static_cast<std::size_t>(nnzb_) * bs_ * bs_;
    if (precision_ == CFDG_PREC_MIXED) {
        std::vector<float> f(v, v + nv);
        cuda_check(cudaMemcpyAsync(vals32_.p, f.data(), nv * sizeof(float), cudaMemcpyHostToDevice, stream_), "H2D");
        cuda_check(cudaStreamSynchronize(stream_), "sync");
    } else {
        cuda_check(cudaMemcpyAsync(vals64_.p, v, nv * sizeof(double), cudaMemcpyHostToDevice, stream_), "H2D");
    }
    lu_ready_ = false;
}

void BsrSystem::get_values_host(double* v) {
    const std::size_t nv = static_cast<std::size_t>(nnzb_) * bs_ * bs_;
    if (precision_ == CFDG_PREC_MIXED) {
        std::vector<float> f(nv);
        cuda_check(cudaMemcpyAsync(f.data(), vals32_.p, nv * sizeof(float), cudaMemcpyDeviceToHost, stream_), "D2H");
        cuda_check(cudaStreamSynchronize(stream_), "sync");
        for (std::size_t i = 0; i < nv; ++i) v[i] = f[i];
    } else {
        cuda_check(cudaMemcpyAsync(v, vals64_.p, nv * sizeof(double), cudaMemcpyDeviceToHost, stream_), "D2H");
        cuda_check(cudaStreamSynchronize(stream_), "sync");
    }
}

// nnzb blocks + columns, row pointers, x and y once, plus the distinct
// vectors read by the fused inner products.
double BsrSystem::spmv_bytes(int n_extra_vectors, bool read_y) const {
    const double sa = (precision_ == CFDG_PREC_MIXED) ? 4.0 : 8.0;
    const double N = double(n_) * bs_;
    return double(nnzb_) * (double(bs_) * bs_ * sa + 4.0) + (n_ + 1.0) * 4.0 + N * 8.0 * (2.0 + (read_y ? 1.0 : 0.0)) +
           N * 8.0 * n_extra_vectors;
}

void BsrSystem::spmv(const double* x, double* y, double alpha, double beta) {
    DotSpec ds{};
    ds.n = 0;
    ProfScope ps(prof_, CFDG_KCAT_SPMV, stream_, 1, spmv_bytes(0, beta != 0.0));
    if (precision_ == CFDG_PREC_MIXED) launch_spmv_ex<float>(view(), vals32_.p, x, y, alpha, beta, ds, nullptr, nullptr, stream_);
    else launch_spmv_ex<double>(view(), vals64_.p, x, y, alpha, beta, ds, nullptr, nullptr, stream_);
    cuda_check(cudaGetLastError(), "spmv launch");
}

// Row groups of the sweep.  LEVEL: level sets of the lower (forward) and
// upper (backward) dependency graphs, so a level-by-level sweep performs
// exactly the arithmetic of the sequential sweep.  COLOR: greedy colouring
// in row order; forward visits colours ascending, backward descending.
void BsrSystem::build_ordering(int ordering) {
    const int32_t n = n_;
    std::vector<int32_t> fwd_key(n, 0), bwd_key(n, 0);
    if (ordering == CFDG_SGS_LEVEL) {
        for (int32_t i = 0; i < n; ++i) {
            int32_t l = 0;
            for (int32_t k = row_ptr_h_[i]; k < row_ptr_h_[i + 1]; ++k) {
                const int32_t j = cols_h_[k];
                if (j < i) l = std::max(l, fwd_key[j] + 1);
            }
            fwd_key[i] = l;
        }
        for (int32_t i = n - 1; i >= 0; --i) {
            int32_t l = 0;
            for (int32_t k = row_ptr_h_[i]; k < row_ptr_h_[i + 1]; ++k) {
                const int32_t j = cols_h_[k];
                if (j > i) l = std::max(l, bwd_key[j] + 1);
            }
            bwd_key[i] = l;
        }
    } else {
        std::vector<int32_t> color(n, -1);
        std::vector<char> used;
        int32_t ncol = 0;
        for (int32_t i = 0; i < n; ++i) {
            used.assign(static_cast<std::size_t>(ncol) + 1, 0);
            for (int32_t k = row_ptr_h_[i]; k < row_ptr_h_[i + 1]; ++k) {
                const int32_t j = cols_h_[k];
                if (j != i && color[j] >= 0) used[color[j]] = 1;
            }
            int32_t c = 0;
            while (used[c]) ++c;
            color[i] = c;
            ncol = std::max(ncol, c + 1);
        }
        for (int32_t i = 0; i < n; ++i) {
            fwd_key[i] = color[i];
            bwd_key[i] = ncol - 1 - color[i];
        }
    }
    auto group = [&](const std::vector<int32_t>& key, std::vector<int32_t>& off, std::vector<int32_t>& rows) {
        int32_t ng = 0;
        for (int32_t i = 0; i < n; ++i) ng = std::max(ng, key[i] + 1);
        off.assign(static_cast<std::size_t>(ng) + 1, 0);
        for (int32_t i = 0; i < n; ++i) ++off[key[i] + 1];
        for (int32_t g = 0; g < ng; ++g) off[g + 1] += off[g];
        rows.resize(n);
        std::vector<int32_t> cur(off.begin(), off.end() - 1);
        for (int32_t i = 0; i < n; ++i) rows[cur[key[i]]++] = i;
    };
    std::vector<int32_t> fr, br;
    group(fwd_key, fwd_off_, fr);
    group(bwd_key, bwd_off_, br);
    // groups whose rows are consecutive (a colour-ordered matrix) run
    // without the row list
    auto contiguous = [&](const std::vector<int32_t>& off, const std::vector<int32_t>& rows,
                          std::vector<int32_t>& first) {
        const int ng = static_cast<int>(off.size()) - 1;
        first.assign(ng, -1);
        for (int g = 0; g < ng; ++g) {
            bool ok = off[g + 1] > off[g];
            for (int32_t q = off[g] + 1; ok && q < off[g + 1]; ++q) ok = rows[q] == rows[q - 1] + 1;
            if (ok) first[g] = rows[off[g]];
        }
    };
    contiguous(fwd_off_, fr, fwd_first_);
    contiguous(bwd_off_, br, bwd_first_);
    // colour-ordered matrix: colour g is rows [fwd_off_[g], fwd_off_[g+1]),
    // so an earlier colour is a smaller row index and the first symmetric
    // sweep can split each row at its diagonal (k_sgs_rows MODE 2 / 3)
    split_ = ordering == CFDG_SGS_COLOR;
    for (std::size_t g = 0; split_ && g < fwd_first_.size(); ++g) split_ = fwd_first_[g] == fwd_off_[g];
    rest_nnzb_ = rest_cols_ = 0.0;
    if (split_ && fwd_off_.size() > 2) {
        std::vector<char> used(n, 0);
        for (int32_t i = fwd_off_[1]; i < n; ++i)
            for (int32_t k = row_ptr_h_[i]; k < row_ptr_h_[i + 1]; ++k) used[cols_h_[k]] = 1;
        for (int32_t j = 0; j < n; ++j) rest_cols_ += used[j];
        rest_nnzb_ = double(nnzb_ - row_ptr_h_[fwd_off_[1]]);
    }
    // Unique-touch bytes of one pass over a group: row list, row pointers,
    // diagonal index, off-diagonal blocks + columns, LU + pivots, r (or the
    // own z read of MODE 3), z write, and each distinct neighbour z block
    // once.  out[0]: full row, out[1]: no neighbours, out[2]: the split half
    // (columns below the diagonal forward, above it backward).
    // Kept as (bytes that do not depend on the matrix precision, matrix
    // blocks read) so that a precision switch (set_precision) keeps them right.
    auto pass_bytes = [&](const std::vector<int32_t>& off, const std::vector<int32_t>& rows, bool lower,
                          std::vector<double>* out, std::vector<double>* blocks) {
        const int ng = static_cast<int>(off.size()) - 1;
        for (int m = 0; m < 3; ++m) {
            out[m].assign(ng, 0.0);
            blocks[m].assign(ng, 0.0);
        }
        std::vector<int32_t> seen(n, -1), seen_half(n, -1);
        for (int g = 0; g < ng; ++g) {
            double offd = 0.0, nbr = 0.0, offd_h = 0.0, nbr_h = 0.0;
            const double R = off[g + 1] - off[g];
            for (int32_t q = off[g]; q < off[g + 1]; ++q) {
                const int32_t i = rows[q];
                offd += row_ptr_h_[i + 1] - row_ptr_h_[i] - 1;
                for (int32_t k = row_ptr_h_[i]; k < row_ptr_h_[i + 1]; ++k) {
                    const int32_t j = cols_h_[k];
                    if (j != i && seen[j] != g) {
                        seen[j] = g;
                        nbr += 1.0;
                    }
                    if (lower ? j < i : j > i) {
                        offd_h += 1.0;
                        if (seen_half[j] != g) {
                            seen_half[j] = g;
                            nbr_h += 1.0;
                        }
                    }
                }
            }
            // list, LU factors + pivots (level) or D^-1 (colour), r, z
            const double own = R * (4.0 + (ordering == CFDG_SGS_COLOR ? 0.0 : bs_) + 2.0 * 8.0 * bs_);
            out[1][g] = own;
            blocks[1][g] = R;
            out[0][g] = own + R * (8.0 + 4.0) + offd * 4.0 + nbr * 8.0 * bs_;
            blocks[0][g] = R + offd;
            out[2][g] = own + R * (8.0 + 4.0) + offd_h * 4.0 + nbr_h * 8.0 * bs_;
            blocks[2][g] = R + offd_h;
        }
    };
    pass_bytes(fwd_off_, fr, true, fwd_bytes_, fwd_blocks_);
    pass_bytes(bwd_off_, br, false, bwd_bytes_, bwd_blocks_);
    upload_or_throw(fwd_rows_, fr, stream_, "sgs rows");
    upload_or_throw(bwd_rows_, br, stream_, "sgs rows");
    upload_or_throw(fwd_off_d_, fwd_off_, stream_, "sgs levels");
    upload_or_throw(bwd_off_d_, bwd_off_, stream_, "sgs levels");
    if (ordering == CFDG_SGS_LEVEL) {
        auto meta = [&](const std::vector<int32_t>& rows) {
            std::vector<int4> m(rows.size());
            for (std::size_t q = 0; q < rows.size(); ++q) {
                const int32_t i = rows[q];
                m[q] = make_int4(i, row_ptr_h_[i], row_ptr_h_[i + 1], diag_h_[i]);
            }
            return m;
        };
        upload_or_throw(fwd_meta_, meta(fr), stream_, "sgs level rows");
        upload_or_throw(bwd_meta_, meta(br), stream_, "sgs level rows");
    }
    cuda_check(cudaStreamSynchronize(stream_), "setup sync");  // the host vectors are rebuilt by the next call
    ordering_ = ordering;
}

void BsrSystem::sgs_setup(int ordering, int sweeps) {
    if (ordering != CFDG_SGS_LEVEL && ordering != CFDG_SGS_COLOR) throw Failure{CFDG_ERR_INVALID, "unknown SGS ordering"};
    if (sweeps < 1) throw Failure{CFDG_ERR_INVALID, "SGS sweeps must be >= 1"};
    if (ordering != ordering_) build_ordering(ordering);
    sweeps_ = sweeps;
    const std::size_t nb2 = static_cast<std::size_t>(n_) * bs_ * bs_;
    if (!piv_.p && n_ > 0) alloc_or_throw(piv_, static_cast<std::size_t>(n_) * bs_, "pivots");
    cuda_check(cudaMemsetAsync(err_.p, 0, sizeof(int), stream_), "memset");
    if (precision_ == CFDG_PREC_MIXED) {
        if (!lu32_.p && n_ > 0) alloc_or_throw(lu32_, nb2, "lu");
        ProfScope ps(prof_, CFDG_KCAT_LU, stream_, 1, double(n_) * (bs_ * bs_ * 8.0 + bs_ + 4.0));
        launch_lu_setup<float>(view(), vals32_.p, lu32_.p, piv_.p, err_.p, ordering_ == CFDG_SGS_COLOR, stream_);
    } else {
        if (!lu64_.p && n_ > 0) alloc_or_throw(lu64_, nb2, "lu");
        ProfScope ps(prof_, CFDG_KCAT_LU, stream_, 1, double(n_) * (bs_ * bs_ * 16.0 + bs_ + 4.0));
        launch_lu_setup<double>(view(), vals64_.p, lu64_.p, piv_.p, err_.p, ordering_ == CFDG_SGS_COLOR, stream_);
    }
    cuda_check(cudaGetLastError(), "lu launch");
    int err = 0;
    cuda_check(cudaMemcpyAsync(&err, err_.p, sizeof(int), cudaMemcpyDeviceToHost, stream_), "D2H");
    cuda_check(cudaStreamSynchronize(stream_), "lu sync");
    if (err > 0) {
        throw Failure{CFDG_ERR_SINGULAR, "SgsPreconditioner: singular diagonal block at row " + std::to_string(err - 1)};
    }
    if (err < 0) {
        throw Failure{CFDG_ERR_NONFINITE, "SgsPreconditioner: non-finite diagonal block at row " + std::to_string(-err - 1)};
    }
    lu_ready_ = true;
}

template <typename MT>
void BsrSystem::sgs_apply_t(const MT* vals, const MT* lu, const double* r, double* z, const int* active,
                            bool skip_last) {
    const BsrView A = view();
    const int nf = groups_fwd(), nbk = groups_bwd();
    const bool color = ordering_ == CFDG_SGS_COLOR;
    // Neighbours ahead of the cursor must read zero on the first forward
    // sweep; with two colours every neighbour of the second colour is of the
    // first colour, and the split sweep never reads them, so no clearing is
    // needed then.
    if (!color || (nf > 2 && !split_)) {
        ProfScope ps(prof_, CFDG_KCAT_SGS, stream_, 0, 8.0 * n_ * bs_);
        cuda_check(cudaMemsetAsync(z, 0, sizeof(double) * static_cast<std::size_t>(n_) * bs_, stream_), "memset");
    }
    for (int sw = 0; sw < sweeps_; ++sw) {
        const bool split = split_ && sw == 0;
        if (!color && level_coop_) {
            // the whole symmetric sweep as one cooperative launch
            double bytes = 0.0;
            for (int g = 0; g < nf; ++g) bytes += fwd_bytes_[0][g] + fwd_blocks_[0][g] * block_bytes();
            for (int g = 0; g < nbk; ++g) bytes += bwd_bytes_[0][g] + bwd_blocks_[0][g] * block_bytes();
            ProfScope ps(prof_, CFDG_KCAT_SGS, stream_, 1, bytes);
            if (fwd_meta_.p &&
                launch_sgs_level_coop<MT>(A, vals, lu, piv_.p, fwd_meta_.p, fwd_off_d_.p, nf, bwd_meta_.p,
                                          bwd_off_d_.p, nbk, r, z, active, stream_))
                continue;
            cudaGetLastError();
            level_coop_ = false;  // level by level from here on
            --prof_->launches;
        }
        for (int g = 0; g < nf; ++g) {
            int mode = 0;
            if (color) {
                if (sw > 0 && g == 0) continue;  // equal to the last backward colour pass
                if (sw == 0) mode = (g == 0) ? 1 : (split ? 2 : 0);  // colour 0: all neighbours still zero
            }
            ProfScope ps(prof_, CFDG_KCAT_SGS, stream_, 1, fwd_bytes_[mode][g] + fwd_blocks_[mode][g] * block_bytes());
            const bool cg = fwd_first_[g] >= 0;
            launch_sgs_rows_ex<MT>(A, vals, lu, piv_.p, cg ? nullptr : fwd_rows_.p + fwd_off_[g], cg ? fwd_first_[g] : 0,
                                   fwd_off_[g + 1] - fwd_off_[g], r, z, mode, color, active, stream_);
        }
        for (int g = 0; g < nbk; ++g) {
            if (color && g == 0) continue;  // first backward colour == last forward colour
            if (skip_last && g == nbk - 1) continue;  // fused with the product (sgs_apply_spmv)
            ProfScope ps(prof_, CFDG_KCAT_SGS, stream_, 1,
                         bwd_bytes_[split ? 2 : 0][g] + bwd_blocks_[split ? 2 : 0][g] * block_bytes());
            const bool cg = bwd_first_[g] >= 0;
            launch_sgs_rows_ex<MT>(A, vals, lu, piv_.p, cg ? nullptr : bwd_rows_.p + bwd_off_[g], cg ? bwd_first_[g] : 0,
                                   bwd_off_[g + 1] - bwd_off_[g], r, z, split ? 3 : 0, color, active, stream_);
        }
    }
}

int BsrSystem::sgs_apply_spmv(const double* r, double* z, double* y, const DotSpec& ds, double* partials,
                              const int* active) {
    if (!lu_ready_) throw Failure{CFDG_ERR_INVALID, "SgsPreconditioner: setup() was not called"};
    const BsrView A = view();
    const bool mixed = precision_ == CFDG_PREC_MIXED;
    const double sa = mixed ? 4.0 : 8.0;
    const double b2 = double(bs_) * bs_;
    const int nx = ds.n == 1 ? 1 : 2;  // vectors the dots read besides y (r0; r0 and s)
    if (!fuse_last_spmv()) {
        sgs_apply(r, z, active);
        ProfScope ps(prof_, CFDG_KCAT_SPMV, stream_, 1, spmv_bytes(nx, false));
        if (mixed) launch_spmv_ex<float>(A, vals32_.p, z, y, 1.0, 0.0, ds, partials, active, stream_);
        else launch_spmv_ex<double>(A, vals64_.p, z, y, 1.0, 0.0, ds, partials, active, stream_);
        cuda_check(cudaGetLastError(), "spmv launch");
        return spmv_blocks(n_, bs_);
    }
    if (mixed) sgs_apply_t<float>(vals32_.p, lu32_.p, r, z, active, true);
    else sgs_apply_t<double>(vals64_.p, lu64_.p, r, z, active, true);
    const int32_t n0 = fwd_off_[1];  // colour 0: rows [0, n0)
    const int g0 = sgs_last_spmv_blocks(n0, bs_);
    {
        const double N0 = double(n0) * bs_;
        ProfScope ps(prof_, CFDG_KCAT_SGS, stream_, 1,
                     bwd_bytes_[2][groups_bwd() - 1] + bwd_blocks_[2][groups_bwd() - 1] * block_bytes() +
                         double(n0) * b2 * sa + N0 * 8.0 * (1.0 + nx));
        if (mixed) launch_sgs_last_spmv<float>(A, vals32_.p, lu32_.p, n0, z, y, ds, partials, active, stream_);
        else launch_sgs_last_spmv<double>(A, vals64_.p, lu64_.p, n0, z, y, ds, partials, active, stream_);
    }
    double* rest = partials + static_cast<std::size_t>(g0) * ds.n;
    {
        const double Nr = double(n_ - n0) * bs_;
        ProfScope ps(prof_, CFDG_KCAT_SPMV, stream_, 1,
                     rest_nnzb_ * (b2 * sa + 4.0) + (n_ - n0 + 1.0) * 4.0 + rest_cols_ * bs_ * 8.0 + Nr * 8.0 * (1.0 + nx));
        if (mixed) launch_spmv_ex<float>(A, vals32_.p, z, y, 1.0, 0.0, ds, rest, active, stream_, n0);
        else launch_spmv_ex<double>(A, vals64_.p, z, y, 1.0, 0.0, ds, rest, active, stream_, n0);
    }
    cuda_check(cudaGetLastError(), "sgs+spmv launch");
    return g0 + spmv_blocks(n_ - n0, bs_);
}

void BsrSystem::sgs_apply(const double* r, double* z, const int* active) {
    if (!lu_ready_) throw Failure{CFDG_ERR_INVALID, "SgsPreconditioner: setup() was not called"};
    if (precision_ == CFDG_PREC_MIXED) sgs_apply_t<float>(vals32_.p, lu32_.p, r, z, active);
    else sgs_apply_t<double>(vals64_.p, lu64_.p, r, z, active);
    cuda_check(cudaGetLastError(), "sgs launch");
}

// The device loop: a graph holding one conditional while-node whose body is
// one captured BiCGSTAB iteration followed by k_krylov_cond.  Captured once
// per (preconditioner, x, b, SGS ordering and sweeps) and relaunched; a
// capture or instantiation error leaves the host loop in charge.
template <typename F>
bool BsrSystem::device_loop_ready(int precond, double* x, const double* b, F&& iteration) {
    const LoopKey key{precond, x, b, ordering_, sweeps_, precision_};
    if (loop_exec_ && key == loop_key_) return true;
    if (loop_failed_) return false;
    release_device_loop();
    cudaGraph_t g = nullptr, body = nullptr;
    const int64_t launches0 = prof_->launches;
    bool capturing = false;
    try {
        cuda_check(cudaGraphCreate(&g, 0), "graph create");
        cuda_check(cudaGraphConditionalHandleCreate(&loop_handle_, g, 1, cudaGraphCondAssignDefault), "graph handle");
        cudaGraphNodeParams cp{};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = loop_handle_;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        cuda_check(cudaGraphAddNode(&node, g, nullptr, 0, &cp), "graph conditional node");
        body = cp.conditional.phGraph_out[0];
        cuda_check(cudaStreamBeginCaptureToGraph(stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
                   "graph capture");
        capturing = true;
        iteration();
        launch_krylov_cond(ks_.p, loop_handle_, stream_);
        ++prof_->launches;
        capturing = false;
        cuda_check(cudaStreamEndCapture(stream_, &body), "graph capture end");
        cuda_check(cudaGraphInstantiate(&loop_exec_, g, 0), "graph instantiate");
    } catch (const Failure&) {
        if (capturing) {
            cudaGraph_t dead = nullptr;
            cudaStreamEndCapture(stream_, &dead);
        }
        cudaGetLastError();
        loop_exec_ = nullptr;
        loop_failed_ = true;
    }
    loop_body_launches_ = prof_->launches - launches0;
    prof_->launches = launches0;
    if (g) cudaGraphDestroy(g);
    if (!loop_exec_) return false;
    loop_key_ = key;
    return true;
}

void BsrSystem::release_device_loop() {
    if (loop_exec_) cudaGraphExecDestroy(loop_exec_);
    loop_exec_ = nullptr;
}

cfdg_krylov_result BsrSystem::bicgstab(int precond, double rel_tol, double abs_tol, int max_it, double* x,
                                       const double* b, bool guess) {
    if (precond == CFDG_PC_SGS && !lu_ready_) throw Failure{CFDG_ERR_INVALID, "SGS preconditioner not set up"};
    const int64_t N = int64_t(n_) * bs_;
    const BsrView A = view();
    const bool mixed = precision_ == CFDG_PREC_MIXED;
    KrylovScalars init{};
    init.max_it = max_it;
    init.rel_tol = rel_tol;
    init.abs_tol = abs_tol;
    init.guess = guess ? 1 : 0;
    cuda_check(cudaMemcpyAsync(ks_.p, &init, sizeof(init), cudaMemcpyHostToDevice, stream_), "H2D");
    const int* active = &ks_.p->state;
    const bool matrix_free = static_cast<bool>(product_);
    // y = A x (or the matrix-free product) with the dots ds; returns the partial rows
    auto spmv_dots = [&](const double* xin, double* yout, const DotSpec& ds) -> int {
        if (matrix_free) return product_(xin, yout, ds, partials_.p, active);
        ProfScope ps(prof_, CFDG_KCAT_SPMV, stream_, 1, spmv_bytes(ds.n == 1 ? 1 : 2, false));
        if (mixed) launch_spmv_ex<float>(A, vals32_.p, xin, yout, 1.0, 0.0, ds, partials_.p, active, stream_);
        else launch_spmv_ex<double>(A, vals64_.p, xin, yout, 1.0, 0.0, ds, partials_.p, active, stream_);
        return spmv_blocks(n_, bs_);
    };
    // r = b - A x; r0 = r; p = r
    {
        DotSpec none{};
        none.n = 0;
        if (matrix_free) {
            if (guess) {
                product_(x, v_.p, none, nullptr, nullptr);
            } else {  // x = 0: A x = 0 without a residual evaluation
                ProfScope ps(prof_, CFDG_KCAT_KRYLOV, stream_, 1, 8.0 * N);
                cuda_check(cudaMemsetAsync(v_.p, 0, sizeof(double) * N, stream_), "memset");
            }
        } else {
            ProfScope ps(prof_, CFDG_KCAT_SPMV, stream_, 1, spmv_bytes(0, false));
            if (mixed) launch_spmv_ex<float>(A, vals32_.p, x, v_.p, 1.0, 0.0, none, nullptr, nullptr, stream_);
            else launch_spmv_ex<double>(A, vals64_.p, x, v_.p, 1.0, 0.0, none, nullptr, nullptr, stream_);
        }
        ProfScope ps(prof_, CFDG_KCAT_KRYLOV, stream_, 2, 5.0 * 8.0 * N);
        launch_krylov_init(N, b, v_.p, r_.p, r0_.p, p_.p, partials_.p, ks_.p, stream_);
        if (guess) {
            ++prof_->launches;
            launch_krylov_guess_reset(N, ks_.p, b, x, r_.p, r0_.p, p_.p, stream_);
        }
    }
    const int nblk = spmv_blocks(n_, bs_);
    const int nvec = dot_blocks(N);
    // One BiCGSTAB iteration (bicgstab.cpp:84-176); every kernel is gated by
    // the device-side state, so a launch after convergence does nothing.
    auto iteration = [&]() {
        {
            ProfScope ps(prof_, CFDG_KCAT_KRYLOV, stream_);
            launch_krylov_begin(ks_.p, stream_);
        }
        DotSpec d1{};
        d1.n = 1;
        d1.a[0] = r0_.p;
        d1.b[0] = nullptr;
        double* phat = p_.p;
        int nb1 = nblk;
        if (precond == CFDG_PC_SGS && matrix_free) {
            sgs_apply(p_.p, phat_.p, active);
            phat = phat_.p;
            nb1 = spmv_dots(phat, v_.p, d1);
        } else if (precond == CFDG_PC_SGS) {
            nb1 = sgs_apply_spmv(p_.p, phat_.p, v_.p, d1, partials_.p, active);
            phat = phat_.p;
        } else {
            nb1 = spmv_dots(phat, v_.p, d1);
        }
        {
            ProfScope ps(prof_, CFDG_KCAT_KRYLOV, stream_, 2, 3.0 * 8.0 * N);
            launch_krylov_gamma(ks_.p, partials_.p, nb1, stream_);
            launch_krylov_s(N, ks_.p, r_.p, v_.p, s_.p, stream_);
        }
        DotSpec d5{};
        d5.n = 5;
        d5.a[0] = nullptr; d5.b[0] = nullptr;   // t.t
        d5.a[1] = nullptr; d5.b[1] = s_.p;      // t.s
        d5.a[2] = r0_.p;   d5.b[2] = nullptr;   // r0.t
        d5.a[3] = r0_.p;   d5.b[3] = s_.p;      // r0.s
        d5.a[4] = s_.p;    d5.b[4] = s_.p;      // s.s
        double* shat = s_.p;
        int nb5 = nblk;
        if (precond == CFDG_PC_SGS && matrix_free) {
            sgs_apply(s_.p, shat_.p, active);
            shat = shat_.p;
            nb5 = spmv_dots(shat, t_.p, d5);
        } else if (precond == CFDG_PC_SGS) {
            nb5 = sgs_apply_spmv(s_.p, shat_.p, t_.p, d5, partials_.p, active);
            shat = shat_.p;
        } else {
            nb5 = spmv_dots(shat, t_.p, d5);
        }
        {
            ProfScope ps(prof_, CFDG_KCAT_KRYLOV, stream_, 3, 10.0 * 8.0 * N);
            launch_krylov_omega(ks_.p, partials_.p, nb5, stream_);
            launch_krylov_update(N, ks_.p, x, phat, shat, s_.p, t_.p, r_.p, p_.p, v_.p, partials_.p, stream_);
            launch_krylov_post(ks_.p, partials_.p, nvec, stream_);
        }
    };
    if (device_loop && !matrix_free && !prof_->on() && max_it > 0 && device_loop_ready(precond, x, b, iteration)) {
        cuda_check(cudaGraphLaunch(loop_exec_, stream_), "krylov graph launch");
        cuda_check(cudaMemcpyAsync(ks_host_, ks_.p, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, stream_), "D2H");
        cuda_check(cudaStreamSynchronize(stream_), "krylov sync");
        prof_->launches += loop_body_launches_ * ks_host_->body_runs;
    } else {
        int it = 0;
        bool done = false;
        while (!done && it < max_it) {
            iteration();
            ++it;
            if (it % check_every == 0 || it == max_it) {
                cuda_check(cudaMemcpyAsync(ks_host_, ks_.p, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, stream_),
                           "D2H");
                cuda_check(cudaStreamSynchronize(stream_), "krylov sync");
                if (ks_host_->state != KS_RUNNING) done = true;
            }
        }
    }
    {
        ProfScope ps(prof_, CFDG_KCAT_KRYLOV, stream_);
        launch_krylov_begin(ks_.p, stream_);  // marks max-iterations when still running
    }
    cuda_check(cudaGetLastError(), "krylov launch");
    cuda_check(cudaMemcpyAsync(ks_host_, ks_.p, sizeof(KrylovScalars), cudaMemcpyDeviceToHost, stream_), "D2H");
    cuda_check(cudaStreamSynchronize(stream_), "krylov sync");
    last_guess_ = guess ? ks_host_->guess : 0;
    last_bnorm_ = ks_host_->bnorm;
    cfdg_krylov_result res{};
    switch (ks_host_->state) {
        case KS_CONVERGED: res.status = CFDG_KRYLOV_CONVERGED; break;
        case KS_DIVERGED: res.status = CFDG_KRYLOV_DIVERGED; break;
        default: res.status = CFDG_KRYLOV_MAX_ITERATIONS; break;
    }
    if (max_it <= 0 && ks_host_->state == KS_RUNNING) res.status = CFDG_KRYLOV_MAX_ITERATIONS;
    res.iterations = ks_host_->it;
    res.initial_residual = ks_host_->initial;
    res.final_residual = ks_host_->rnorm;
    return res;
}

void BsrSystem::gm_alloc(int restart) {
    if (gm_restart_ == restart) return;
    const std::size_t N = static_cast<std::size_t>(n_) * bs_;
    gm_V_.release();
    alloc_or_throw(gm_V_, N * (restart + 1), "GMRES basis");
    alloc_or_throw(gm_z_, N, "GMRES vector");
    alloc_or_throw(gm_part_, static_cast<std::size_t>(gm_partial_blocks(int64_t(N))) * gm_chunk() + 8, "GMRES partials");
    alloc_or_throw(gm_h_, 3 * static_cast<std::size_t>(restart + 1) + 8, "GMRES coefficients");
    cuda_check(cudaMemsetAsync(gm_h_.p, 0, gm_h_.count * sizeof(double), stream_), "memset");
    if (gm_h_host_) cudaFreeHost(gm_h_host_);
    gm_h_host_ = nullptr;
    cuda_check(cudaMallocHost(reinterpret_cast<void**>(&gm_h_host_), sizeof(double) * (3 * (restart + 1) + 8)),
               "cudaMallocHost");
    gm_restart_ = restart;
}

// GMRES(m) with right preconditioning (Saad, Iterative Methods for Sparse
// Linear Systems, 2nd ed., Alg. 9.5): Arnoldi on A M^-1 by classical
// Gram-Schmidt with one reorthogonalisation pass, Givens rotations of the
// Hessenberg column on the host (one coefficient read per iteration), the
// update x += M^-1 V y at the end of each cycle and the true residual at
// each restart.  The residual estimate |g_{j+1}| decreases monotonically.
cfdg_krylov_result BsrSystem::gmres(int precond, double rel_tol, double abs_tol, int max_it, int restart, double* x,
                                    const double* b, bool guess) {
    if (precond == CFDG_PC_SGS && !lu_ready_) throw Failure{CFDG_ERR_INVALID, "SGS preconditioner not set up"};
    if (restart < 1 || restart > 200) throw Failure{CFDG_ERR_INVALID, "GMRES restart must be in [1, 200]"};
    gm_alloc(restart);
    const int64_t N = int64_t(n_) * bs_;
    const BsrView A = view();
    const bool mixed = precision_ == CFDG_PREC_MIXED;
    const int m = restart;
    double* V = gm_V_.p;
    double* hd = gm_h_.p;        // [0, m+1) first projection, [m+1, 2m+2) second, [2m+2] |w|^2
    double* hh = gm_h_host_;
    DotSpec none{};
    none.n = 0;
    auto vec = [&](int k) { return V + int64_t(k) * N; };
    auto apply_A = [&](const double* xin, double* yout) {
        if (product_) {
            product_(xin, yout, none, nullptr, nullptr);
            return;
        }
        ProfScope ps(prof_, CFDG_KCAT_SPMV, stream_, 1, spmv_bytes(0, false));
        if (mixed) launch_spmv_ex<float>(A, vals32_.p, xin, yout, 1.0, 0.0, none, nullptr, nullptr, stream_);
        else launch_spmv_ex<double>(A, vals64_.p, xin, yout, 1.0, 0.0, none, nullptr, nullptr, stream_);
    };
    auto precond_apply = [&](const double* r, double* z) {
        if (precond == CFDG_PC_SGS) {
            sgs_apply(r, z, nullptr);
        } else {
            ProfScope ps(prof_, CFDG_KCAT_KRYLOV, stream_, 1, 16.0 * N);
            cuda_check(cudaMemcpyAsync(z, r, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream_), "D2D");
        }
    };
    const int chunk = gm_chunk();
    auto dots = [&](int kn, const double* w, double* h) {
        ProfScope ps(prof_, CFDG_KCAT_KRYLOV, stream_, 2 * ((kn + chunk - 1) / chunk),
                     8.0 * N * (kn + (kn + chunk - 1) / chunk));
        launch_gm_dots(N, V, N, 0, kn, w, gm_part_.p, h, stream_);
    };
    auto norm2 = [&](const double* w, double* h) {
        ProfScope ps(prof_, CFDG_KCAT_KRYLOV, stream_, 2, 8.0 * N);
        launch_gm_dots(N, w, 0, 0, 1, w, gm_part_.p, h, stream_);
    };
    auto read_h = [&](int count) {
        cuda_check(cudaMemcpyAsync(hh, hd, sizeof(double) * count, cudaMemcpyDeviceToHost, stream_), "D2H");
        cuda_check(cudaStreamSynchronize(stream_), "gmres sync");
    };
    auto axpy = [&](double a, const double* xin, double* y, bool acc) {
        ProfScope ps(prof_, CFDG_KCAT_KRYLOV, stream_, 1, 8.0 * N * (acc ? 3.0 : 2.0));
        launch_gm_axpy(N, a, xin, y, acc, stream_);
    };
    // r0 = b - A x in V_0; ||b||
    norm2(b, hd + 2 * m + 2);
    read_h(2 * m + 3);
    const double bnorm = std::sqrt(hh[2 * m + 2]);
    double beta = bnorm;
    int guess_state = 0;
    // x holds x0; with the matrix-free product and no guess the caller has
    // zeroed it, and r0 = b needs no residual evaluation
    bool zero_start = product_ && !guess;
    if (!zero_start) {
        apply_A(x, vec(0));
        axpy(-1.0, vec(0), vec(0), false);
        axpy(1.0, b, vec(0), true);
        norm2(vec(0), hd + 2 * m + 2);
        read_h(2 * m + 3);
        beta = std::sqrt(hh[2 * m + 2]);
        if (guess) {
            guess_state = 1;
            if (!(beta < bnorm)) {  // the guess does not beat x = 0
                guess_state = 2;
                beta = bnorm;
                zero_start = true;
            }
        }
    }
    if (zero_start) {
        cuda_check(cudaMemsetAsync(x, 0, sizeof(double) * N, stream_), "memset");
        cuda_check(cudaMemcpyAsync(vec(0), b, sizeof(double) * N, cudaMemcpyDeviceToDevice, stream_), "D2D");
    }
    const double tol = std::max(abs_tol, rel_tol * (bnorm > 0.0 ? bnorm : 1.0));
    cfdg_krylov_result res{};
    res.initial_residual = beta;
    res.final_residual = beta;
    int its = 0;
    int state = std::isfinite(beta) ? (beta <= tol ? KS_CONVERGED : KS_RUNNING) : KS_DIVERGED;
    std::vector<double> R(static_cast<std::size_t>(m) * m), g(m + 1), cs(m), sn(m), y(m);
    while (state == KS_RUNNING) {
        axpy(1.0 / beta, vec(0), vec(0), false);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int k = 0;
        double resid = beta;
        for (int j = 0; j < m && its < max_it; ++j) {
            double* w = vec(j + 1);
            precond_apply(vec(j), gm_z_.p);
            apply_A(gm_z_.p, w);
            dots(j + 1, w, hd);
            {
                ProfScope ps(prof_, CFDG_KCAT_KRYLOV, stream_, 1, 8.0 * N * (j + 3));
                launch_gm_update(N, V, N, j + 1, hd, w, true, stream_);
            }
            dots(j + 1, w, hd + m + 1);
            {
                ProfScope ps(prof_, CFDG_KCAT_KRYLOV, stream_, 1, 8.0 * N * (j + 3));
                launch_gm_update(N, V, N, j + 1, hd + m + 1, w, true, stream_);
            }
            norm2(w, hd + 2 * m + 2);
            read_h(2 * m + 3);
            ++its;
            double col[201];
            for (int i = 0; i <= j; ++i) col[i] = hh[i] + hh[m + 1 + i];
            const double hn = std::sqrt(std::max(hh[2 * m + 2], 0.0));
            col[j + 1] = hn;
            for (int i = 0; i < j; ++i) {  // previous rotations
                const double t = cs[i] * col[i] + sn[i] * col[i + 1];
                col[i + 1] = -sn[i] * col[i] + cs[i] * col[i + 1];
                col[i] = t;
            }
            const double rr = std::hypot(col[j], col[j + 1]);
            if (!(rr > 0.0) || !std::isfinite(rr)) {
                state = KS_DIVERGED;
                break;
            }
            cs[j] = col[j] / rr;
            sn[j] = col[j + 1] / rr;
            col[j] = rr;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            for (int i = 0; i <= j; ++i) R[static_cast<std::size_t>(i) * m + j] = col[i];
            k = j + 1;
            resid = std::fabs(g[j + 1]);
            if (resid <= tol || hn == 0.0) {
                state = KS_CONVERGED;
                break;
            }
            axpy(1.0 / hn, w, w, false);
        }
        if (k > 0) {
            // y = R^-1 g, x += M^-1 (V y)
            for (int i = k - 1; i >= 0; --i) {
                double s = g[i];
                for (int l = i + 1; l < k; ++l) s -= R[static_cast<std::size_t>(i) * m + l] * y[l];
                y[i] = s / R[static_cast<std::size_t>(i) * m + i];
            }
            cuda_check(cudaMemcpyAsync(hd, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, stream_), "H2D");
            {
                ProfScope ps(prof_, CFDG_KCAT_KRYLOV, stream_, 1, 8.0 * N * (k + 1));
                launch_gm_update(N, V, N, k, hd, gm_z_.p, false, stream_);
            }
            precond_apply(gm_z_.p, vec(k));
            axpy(1.0, vec(k), x, true);
            cuda_check(cudaStreamSynchronize(stream_), "gmres sync");  // y on the host stays alive until here
        }
        res.final_residual = resid;
        if (state != KS_RUNNING) break;
        if (its >= max_it) {
            state = KS_MAXIT;
            break;
        }
        // restart from the true residual
        apply_A(x, vec(0));
        axpy(-1.0, vec(0), vec(0), false);
        axpy(1.0, b, vec(0), true);
        norm2(vec(0), hd + 2 * m + 2);
        read_h(2 * m + 3);
        beta = std::sqrt(hh[2 * m + 2]);
        res.final_residual = beta;
        if (!std::isfinite(beta)) state = KS_DIVERGED;
        else if (beta <= tol) state = KS_CONVERGED;
    }
    cuda_check(cudaGetLastError(), "gmres launch");
    last_guess_ = guess ? guess_state : 0;
    last_bnorm_ = bnorm;
    switch (state) {
        case KS_CONVERGED: res.status = CFDG_KRYLOV_CONVERGED; break;
        case KS_DIVERGED: res.status = CFDG_KRYLOV_DIVERGED; break;
        default: res.status = CFDG_KRYLOV_MAX_ITERATIONS; break;
    }
    res.iterations = its;
    return res;
}

// ================================================================= Solver
Solver::Solver(int device, const cfdg_mesh_host& mesh, const cfdg_config& cfg, const cfdg_bc_desc* bcs, int n_bcs)
    : device_(device), cfg_(cfg) {
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
    gas_.gamma = cfg.gamma;
    gas_.R = cfg.gas_constant;
    gas_.cv = cfg.gas_constant / (cfg.gamma - 1.0);
    gas_.cp = cfg.gamma * gas_.cv;
    gas_.prandtl = cfg.prandtl;
    gas_.prandtl_turb = cfg.prandtl_turb;
    sa_ = cfg.turbulence == 1;
    if (sa_ && !cfg.viscous) throw Failure{CFDG_ERR_INVALID, "Spalart-Allmaras needs the viscous equations"};
    nv_ = sa_ ? 6 : 5;
    if (cfg.jacobian != CFDG_JAC_REFERENCE && cfg.jacobian != CFDG_JAC_THIN_LAYER)
        throw Failure{CFDG_ERR_INVALID, "unknown Jacobian variant"};
    if (cfg.krylov_loop != CFDG_KRYLOV_DEVICE_LOOP && cfg.krylov_loop != CFDG_KRYLOV_HOST_LOOP)
        throw Failure{CFDG_ERR_INVALID, "unknown Krylov loop driver"};
    if (cfg.pre_freeze != CFDG_PREFREEZE_CONFIGURED && cfg.pre_freeze != CFDG_PREFREEZE_FP64)
        throw Failure{CFDG_ERR_INVALID, "unknown pre-freeze mode"};
    if (cfg.time_mode != CFDG_TIME_STEADY && cfg.time_mode != CFDG_TIME_UNSTEADY)
        throw Failure{CFDG_ERR_INVALID, "unknown time mode"};
    if (cfg.newton_operator != CFDG_NEWTON_PICARD && cfg.newton_operator != CFDG_NEWTON_JACOBIAN_FREE)
        throw Failure{CFDG_ERR_INVALID, "unknown Newton operator"};
    if (cfg.newton_operator == CFDG_NEWTON_JACOBIAN_FREE &&
        (!(cfg.jf_eps > 0.0) || !(cfg.jf_rel_tol > 0.0) || cfg.jf_max_iterations < 1 || !(cfg.jf_max_change >= 0.0) ||
         !(cfg.jf_accept > 0.0 && cfg.jf_accept <= 1.0)))
        throw Failure{CFDG_ERR_INVALID, "Jacobian-free Newton needs jf_eps > 0, jf_rel_tol > 0, jf_max_iterations >= 1, "
                                        "jf_max_change >= 0, 0 < jf_accept <= 1"};
    if (cfg.newton_operator == CFDG_NEWTON_JACOBIAN_FREE &&
        ((cfg.jf_krylov != CFDG_JF_BICGSTAB && cfg.jf_krylov != CFDG_JF_GMRES) ||
         (cfg.jf_krylov == CFDG_JF_GMRES && (cfg.jf_restart < 1 || cfg.jf_restart > 200))))
        throw Failure{CFDG_ERR_INVALID, "jf_krylov must be CFDG_JF_BICGSTAB or CFDG_JF_GMRES with jf_restart in [1, 200]"};
    unsteady_ = cfg.time_mode == CFDG_TIME_UNSTEADY;
    if (unsteady_ && (cfg.bdf_order < 1 || cfg.bdf_order > 2 || !(cfg.dt_physical > 0.0) || cfg.max_time_steps < 0))
        throw Failure{CFDG_ERR_INVALID, "unsteady mode needs bdf_order 1 or 2, dt_physical > 0, max_time_steps >= 0"};
    muscl_ = cfg.reconstruction == CFDG_RECON_MUSCL;
    need_grad_ = muscl_ || cfg.viscous;
    if (cfg.gradient != CFDG_GRAD_LSQ_FACE && cfg.gradient != CFDG_GRAD_LSQ_NODE && need_grad_)
        throw Failure{CFDG_ERR_UNSUPPORTED, "gradient operator not built (least-squares face or node only)"};
    cuda_check(cudaMallocHost(reinterpret_cast<void**>(&l2_host_), sizeof(double) * 8), "cudaMallocHost");

    HostMesh hm;
    hm.from_view(mesh);
    if (hm.n_cells <= 0 || hm.n_faces <= 0 || hm.n_inner < 0 || hm.n_inner > hm.n_faces)
        throw Failure{CFDG_ERR_MESH, "empty or inconsistent mesh"};
    for (int32_t f = 0; f < hm.n_faces; ++f) {
        const bool inner = f < hm.n_inner;
        if (hm.owner[f] < 0 || hm.owner[f] >= hm.n_cells) throw Failure{CFDG_ERR_MESH, "face owner out of range"};
        if (inner && (hm.neigh[f] < 0 || hm.neigh[f] >= hm.n_cells)) throw Failure{CFDG_ERR_MESH, "interior face without neighbour"};
        if (!inner && hm.neigh[f] >= 0) throw Failure{CFDG_ERR_MESH, "boundary face with a neighbour (3-zone order broken)"};
        if (!inner && (hm.patch[f] < 0)) throw Failure{CFDG_ERR_MESH, "boundary face without patch"};
        if (!(hm.area[f] > 1e-15)) throw Failure{CFDG_ERR_MESH, "zero-area face"};
    }
    for (int32_t c = 0; c < hm.n_cells; ++c)
        if (!(hm.vol[c] > 1e-15)) throw Failure{CFDG_ERR_MESH, "non-positive cell volume"};
    for (int32_t f = hm.n_inner + 1; f < hm.n_faces; ++f)
        if (hm.patch[f] < hm.patch[f - 1]) throw Failure{CFDG_ERR_MESH, "boundary faces not grouped by patch"};

    setup_mesh(mesh);
    setup_bcs(bcs, n_bcs, hm);
    const Csr c2c = build_cell_cells_face(hm);
    setup_matrix(hm, c2c);
    sys_->set_profiler(&prof_);
    {
        const Csr c2f = build_cell_faces(hm);
        const int64_t E = need_grad_ ? g_entries_ : 0;
        compute_alg_bytes(E, static_cast<int64_t>(c2c.val.size()), static_cast<int64_t>(c2f.val.size()));
    }
    if (sa_) setup_sa(hm);
    cuda_check(cudaStreamSynchronize(stream_), "setup sync");
}

Solver::~Solver() {
    if (l2_host_) cudaFreeHost(l2_host_);
    if (jf_host_) cudaFreeHost(jf_host_);
    sys_.reset();
    if (stream_) cudaStreamDestroy(stream_);
}

void Solver::setup_mesh(const cfdg_mesh_host& mesh) {
    HostMesh hm;
    hm.from_view(mesh);
    const int32_t n = hm.n_cells, nf = hm.n_faces, ni = hm.n_inner, nb = nf - ni;
    dm_.n = n;
    dm_.nf = nf;
    dm_.ni = ni;
    dm_.nb = nb;
    dm_.nt = n + nb;
    cudaStream_t s = stream_;
    upload_or_throw(owner_, hm.owner, s, "owner");
    upload_or_throw(neigh_, hm.neigh, s, "neigh");
    std::vector<int32_t> bp(hm.patch.begin() + ni, hm.patch.end());
    upload_or_throw(bpatch_, bp, s, "bpatch");
    upload_or_throw(fnx_, hm.fnx, s, "fnx");
    upload_or_throw(fny_, hm.fny, s, "fny");
    upload_or_throw(fnz_, hm.fnz, s, "fnz");
    upload_or_throw(farea_, hm.area, s, "area");
    upload_or_throw(fcx_, hm.fcx, s, "fcx");
    upload_or_throw(fcy_, hm.fcy, s, "fcy");
    upload_or_throw(fcz_, hm.fcz, s, "fcz");
    upload_or_throw(ccx_, hm.ccx, s, "ccx");
    upload_or_throw(ccy_, hm.ccy, s, "ccy");
    upload_or_throw(ccz_, hm.ccz, s, "ccz");
    upload_or_throw(vol_, hm.vol, s, "vol");
    // face-cell distance vectors (build_face_cell_dist_vectors,
    // src/mesh/aux_geometry.cpp:11-51) and 1/|d| (build_face_cell_dist_inv :107-156)
    std::vector<double> dx(nf), dy(nf), dz(nf), dinv(nf);
    for (int32_t f = 0; f < nf; ++f) {
        const int32_t u = hm.owner[f];
        if (f < ni) {
            const int32_t v = hm.neigh[f];
            dx[f] = hm.ccx[v] - hm.ccx[u];
            dy[f] = hm.ccy[v] - hm.ccy[u];
            dz[f] = hm.ccz[v] - hm.ccz[u];
            const double d = std::sqrt((hm.ccx[v] - hm.ccx[u]) * (hm.ccx[v] - hm.ccx[u]) +
                                       (hm.ccy[v] - hm.ccy[u]) * (hm.ccy[v] - hm.ccy[u]) +
                                       (hm.ccz[v] - hm.ccz[u]) * (hm.ccz[v] - hm.ccz[u]));
            dinv[f] = 1.0 / d;
        } else {
            dx[f] = 2.0 * (hm.fcx[f] - hm.ccx[u]);
            dy[f] = 2.0 * (hm.fcy[f] - hm.ccy[u]);
            dz[f] = 2.0 * (hm.fcz[f] - hm.ccz[u]);
            const double d = std::sqrt(4.0 * (hm.fcx[f] - hm.ccx[u]) * (hm.fcx[f] - hm.ccx[u]) +
                                       4.0 * (hm.fcy[f] - hm.ccy[u]) * (hm.fcy[f] - hm.ccy[u]) +
                                       4.0 * (hm.fcz[f] - hm.ccz[u]) * (hm.fcz[f] - hm.ccz[u]));
            dinv[f] = 1.0 / d;
        }
    }
    upload_or_throw(fdx_, dx, s, "fdx");
    upload_or_throw(fdy_, dy, s, "fdy");
    upload_or_throw(fdz_, dz, s, "fdz");
    upload_or_throw(finv_d_, dinv, s, "finv_d");
    const Csr c2f = build_cell_faces(hm);
    upload_or_throw(c2f_off_, c2f.off, s, "c2f_off");
    upload_or_throw(c2f_, c2f.val, s, "c2f");
    std::vector<int32_t> c2fs(c2f.val.size());
    for (int32_t c = 0; c < n; ++c)
        for (int32_t e = c2f.off[c]; e < c2f.off[c + 1]; ++e)
            c2fs[e] = hm.owner[c2f.val[e]] == c ? c2f.val[e] : ~c2f.val[e];
    upload_or_throw(c2fs_, c2fs, s, "c2fs");
    const Csr c2c = build_cell_cells_face(hm);
    upload_or_throw(c2c_off_, c2c.off, s, "c2c_off");
    upload_or_throw(c2c_, c2c.val, s, "c2c");
    if (need_grad_) {
        const Csr st = (cfg_.gradient == CFDG_GRAD_LSQ_FACE) ? c2c : build_cell_cells_node(hm);
        const LsqSlices sl = build_lsq_slices(hm, st);
        g_entries_ = sl.entries;
        upload_or_throw(g_soff_, sl.soff, s, "g_soff");
        upload_or_throw(g_col_, sl.col, s, "g_col");
        upload_or_throw(g_wx_, sl.wx, s, "g_wx");
        upload_or_throw(g_wy_, sl.wy, s, "g_wy");
        upload_or_throw(g_wz_, sl.wz, s, "g_wz");
        // the host vectors die at scope end: make the copies complete first
        cuda_check(cudaStreamSynchronize(s), "setup sync");
    }
    cuda_check(cudaStreamSynchronize(s), "setup sync");
    dm_.owner = owner_.p;
    dm_.neigh = neigh_.p;
    dm_.bpatch = bpatch_.p;
    dm_.fnx = fnx_.p;
    dm_.fny = fny_.p;
    dm_.fnz = fnz_.p;
    dm_.farea = farea_.p;
    dm_.fcx = fcx_.p;
    dm_.fcy = fcy_.p;
    dm_.fcz = fcz_.p;
    dm_.fdx = fdx_.p;
    dm_.fdy = fdy_.p;
    dm_.fdz = fdz_.p;
    dm_.finv_d = finv_d_.p;
    dm_.ccx = ccx_.p;
    dm_.ccy = ccy_.p;
    dm_.ccz = ccz_.p;
    dm_.vol = vol_.p;
    dm_.c2f_off = c2f_off_.p;
    dm_.c2f = c2f_.p;
    dm_.c2fs = c2fs_.p;
    dm_.c2c_off = c2c_off_.p;
    dm_.c2c = c2c_.p;
    dm_.g_soff = g_soff_.p;
    dm_.g_col = g_col_.p;
    dm_.g_wx = g_wx_.p;
    dm_.g_wy = g_wy_.p;
    dm_.g_wz = g_wz_.p;

    // fields
    const std::size_t nt = static_cast<std::size_t>(dm_.nt), nn = static_cast<std::size_t>(n);
    alloc_or_throw(U_, nn * nv_, "U");
    alloc_or_throw(q_, nt * (sa_ ? 6 : 5), "q");  // with SA, plane 5 holds nu_tilde
    alloc_or_throw(grad_, need_grad_ ? nt * 3 * nv_ : 1, "grad");
    alloc_or_throw(phi_, muscl_ ? nn * 5 : 1, "phi");
    alloc_or_throw(fflux_, static_cast<std::size_t>(nf) * 6, "fflux");
    alloc_or_throw(res_, nn * nv_, "res");
    alloc_or_throw(lam_, nn, "lam");
    alloc_or_throw(dt_, nn, "dt");
    alloc_or_throw(alpha_, nn, "alpha");
    cuda_check(cudaMemsetAsync(q_.p, 0, q_.count * sizeof(double), s), "memset");
    cuda_check(cudaMemsetAsync(grad_.p, 0, grad_.count * sizeof(double), s), "memset");
    cuda_check(cudaMemsetAsync(phi_.p, 0, phi_.count * sizeof(double), s), "memset");
    cuda_check(cudaMemsetAsync(res_.p, 0, res_.count * sizeof(double), s), "memset");
    cuda_check(cudaMemsetAsync(lam_.p, 0, lam_.count * sizeof(double), s), "memset");
    cuda_check(cudaMemsetAsync(dt_.p, 0, dt_.count * sizeof(double), s), "memset");
    cuda_check(cudaMemsetAsync(alpha_.p, 0, alpha_.count * sizeof(double), s), "memset");
    df_.U = U_.p;
    df_.q = q_.p;
    df_.grad = grad_.p;
    df_.phi = phi_.p;
    df_.fflux = fflux_.p;
    df_.res = res_.p;
    df_.lam = lam_.p;
    df_.dt = dt_.p;
    df_.alpha = alpha_.p;
    df_.mut = nullptr;
    alloc_or_throw(norm_partials_, static_cast<std::size_t>(norm_blocks(n)) * 6 + 8, "norm partials");
    alloc_or_throw(l2_, 8, "l2");
}

// Unique-touch byte counts (each array element once per launch, at its
// stored precision) of the residual-side kernels.
void Solver::compute_alg_bytes(int64_t E, int64_t n_c2c, int64_t n_c2f) {
    const double n = dm_.n, nb = dm_.nb, F = dm_.nf, Fi = dm_.ni, d = 8.0, i4 = 4.0;
    const double visc = cfg_.viscous ? 1.0 : 0.0;
    ab_.prim = n * 5 * d * 2 + nb * (5 * d + i4 + 3 * d + 3 * d + i4 + 5 * d) + nb * 3 * d;
    ab_.grad = n * 5 * d + (n + 1) * i4 + double(E) * (i4 + 3 * d) + n * 15 * d;
    // ghost gradients alone (the limiter frozen or not in use)
    ab_.ghost_grad = nb * (15 * d + 5 * d + i4 + i4 + 3 * d + 3 * d + 3 * d);
    ab_.limiter = (muscl_ ? n * (5 + 15 + 3 + 1 + 5) * d + (n + 1) * i4 * 2 + double(n_c2c) * i4 +
                                double(n_c2f) * i4 + F * 3 * d
                          : 0.0) +
                  ab_.ghost_grad;
    ab_.face_flux = F * (2 * i4 + 4 * d + 3 * d) + visc * F * 4 * d + (n + nb) * (5 + 15 + 5 + 3) * d + F * 6 * d;
    ab_.cell_gather = (n + 1) * i4 + double(n_c2f) * i4 + F * 6 * d + n * 6 * d;
    const double b2 = double(nv_) * nv_;
    const double nnzb = sys_ ? double(sys_->nnzb()) : n + 2 * Fi;
    // row-centric assembly: face owner/neigh, normal, area (+ 1/|d|), primitives
    // of cells and ghosts, alpha, CSR cell -> faces, face_pos, diagonal slots,
    // boundary patch ids, the row -> cell map; every block written once
    ab_.jac = F * (2 * i4 + 4 * d + visc * d) + (n + nb) * 5 * d + n * d + (n + 1) * i4 + double(n_c2f) * i4 +
              Fi * 2 * i4 + n * i4 + nb * i4 + n * i4;  // + the block stores, at the stored precision
    ab_.jac_blocks = nnzb * b2;
    ab_.dt_rhs = n * (d * 2 + d * 2 + nv_ * d + nv_ * d);  // lam, vol -> dt, alpha; R -> b
    ab_.state_update = n * nv_ * d * 3;
    ab_.norms = n * nv_ * d;
}

void Solver::setup_bcs(const cfdg_bc_desc* bcs, int n_bcs, const HostMesh& hm) {
    const int np = std::max(hm.n_patches, 1);
    patches_h_.assign(np, BcPatch{});
    for (auto& p : patches_h_) {
        p.kind = -1;
        p.sa_kind = 3;
    }
    for (int i = 0; i < n_bcs; ++i) {
        const cfdg_bc_desc& d = bcs[i];
        if (d.patch_id < 0 || d.patch_id >= np) continue;  // patch absent on this mesh
        if (d.type < 0 || d.type > 8) throw Failure{CFDG_ERR_INVALID, "unknown BC type"};
        BcPatch& P = patches_h_[d.patch_id];
        P = BcPatch{};
        P.kind = d.type;
        switch (d.type) {
            case CFDG_BC_SUPERSONIC_INLET: {
                const Inflow s = resolve_inflow(d, gas_, d.p);
                P.qfix[0] = s.p; P.qfix[1] = s.u; P.qfix[2] = s.v; P.qfix[3] = s.w; P.qfix[4] = s.T;
                P.sa_kind = 1;
                break;
            }
            case CFDG_BC_FARFIELD: {
                const Inflow s = resolve_inflow(d, gas_, d.p);
                P.far_p = s.p; P.far_T = s.T; P.far_u = s.u; P.far_v = s.v; P.far_w = s.w;
                P.sa_kind = 1;
                break;
            }
            case CFDG_BC_NO_SLIP_WALL:
                P.qfix[1] = d.velocity[0]; P.qfix[2] = d.velocity[1]; P.qfix[3] = d.velocity[2]; P.qfix[4] = d.t;
                P.sa_kind = 0;
                break;
            case CFDG_BC_NO_SLIP_WALL_HEAT_FLUX:
                P.qfix[1] = d.velocity[0]; P.qfix[2] = d.velocity[1]; P.qfix[3] = d.velocity[2];
                P.tmp_grad = d.tmp_grad;
                P.sa_kind = 0;
                break;
            case CFDG_BC_SUBSONIC_INLET: {
                const double p_ref = (d.p > 0.0) ? d.p : 101325.0;
                const Inflow s = resolve_inflow(d, gas_, p_ref);
                P.qfix[1] = s.u; P.qfix[2] = s.v; P.qfix[3] = s.w; P.qfix[4] = s.T;
                P.sa_kind = 1;
                break;
            }
            case CFDG_BC_SUBSONIC_OUTLET:
                P.p_out = d.p;
                P.sa_kind = 2;
                break;
            case CFDG_BC_SUPERSONIC_OUTLET:
                P.sa_kind = 2;
                break;
            default:
                P.sa_kind = 3;
                break;
        }
    }
    for (int32_t f = hm.n_inner; f < hm.n_faces; ++f) {
        const int32_t p = hm.patch[f];
        if (p >= np || patches_h_[p].kind < 0)
            throw Failure{CFDG_ERR_INVALID, "boundary patch " + std::to_string(p) + " has no boundary condition"};
    }
    upload_or_throw(patches_, patches_h_, stream_, "patches");
    cuda_check(cudaStreamSynchronize(stream_), "setup sync");
    dm_.patches = patches_.p;
    dm_.n_patches = np;
}

void Solver::setup_matrix(const HostMesh& hm, const Csr& c2c) {
    const int32_t n = hm.n_cells;
    // Multicolour SGS: store the system in colour order (greedy colouring in
    // cell order, as the preconditioner's own), so that every colour pass
    // streams one contiguous range of block rows.  The level-scheduled
    // (parity) ordering keeps the reference's cell order.
    row_of_h_.clear();
    cell_of_h_.clear();
    if (cfg_.precond == CFDG_PC_SGS && cfg_.sgs_ordering == CFDG_SGS_COLOR) {
        std::vector<int32_t> color(static_cast<std::size_t>(n), -1);
        std::vector<char> used;
        int32_t ncol = 0;
        for (int32_t c = 0; c < n; ++c) {
            used.assign(static_cast<std::size_t>(ncol) + 1, 0);
            for (int32_t k = c2c.off[c]; k < c2c.off[c + 1]; ++k) {
                const int32_t j = c2c.val[k];
                if (color[j] >= 0) used[color[j]] = 1;
            }
            int32_t col = 0;
            while (used[col]) ++col;
            color[c] = col;
            ncol = std::max(ncol, col + 1);
        }
        std::vector<int32_t> start(static_cast<std::size_t>(ncol) + 1, 0);
        for (int32_t c = 0; c < n; ++c) ++start[color[c] + 1];
        for (int32_t g = 0; g < ncol; ++g) start[g + 1] += start[g];
        row_of_h_.resize(n);
        cell_of_h_.resize(n);
        for (int32_t c = 0; c < n; ++c) {
            const int32_t r = start[color[c]]++;
            row_of_h_[c] = r;
            cell_of_h_[r] = c;
        }
    }
    const bool perm = !row_of_h_.empty();
    auto R = [&](int32_t c) { return perm ? row_of_h_[c] : c; };
    // bsr_assemble (linalg/bsr_helpers.hpp:16-59): self + face neighbours, sorted.
    std::vector<int32_t> row_ptr(static_cast<std::size_t>(n) + 1, 0), cols;
    cols.reserve(c2c.val.size() + n);
    for (int32_t r = 0; r < n; ++r) {
        const int32_t c = perm ? cell_of_h_[r] : r;
        const std::size_t s0 = cols.size();
        cols.push_back(r);
        for (int32_t k = c2c.off[c]; k < c2c.off[c + 1]; ++k) cols.push_back(R(c2c.val[k]));
        std::sort(cols.begin() + s0, cols.end());
        row_ptr[r + 1] = static_cast<int32_t>(cols.size());
    }
    sys_ = std::make_unique<BsrSystem>(device_, n, nv_, row_ptr.data(), cols.data(),
                                       pre_freeze_phase() ? CFDG_PREC_FP64 : cfg_.precision, stream_);
    sys_->device_loop = cfg_.krylov_loop == CFDG_KRYLOV_DEVICE_LOOP;
    auto pos = [&](int32_t row, int32_t col) -> int32_t {
        const auto b = cols.begin() + row_ptr[row], e = cols.begin() + row_ptr[row + 1];
        const auto it = std::lower_bound(b, e, col);
        if (it == e || *it != col) throw Failure{CFDG_ERR_MESH, "dual graph misses a face neighbour"};
        return static_cast<int32_t>(it - cols.begin());
    };
    std::vector<int32_t> fpos(static_cast<std::size_t>(2) * hm.n_inner);
    for (int32_t f = 0; f < hm.n_inner; ++f) {
        fpos[2 * f] = pos(R(hm.owner[f]), R(hm.neigh[f]));
        fpos[2 * f + 1] = pos(R(hm.neigh[f]), R(hm.owner[f]));
    }
    upload_or_throw(face_pos_, fpos, stream_, "face_pos");
    if (perm) {
        upload_or_throw(row_of_, row_of_h_, stream_, "row_of");
        upload_or_throw(cell_of_, cell_of_h_, stream_, "cell_of");
    }
    dm_.row_of = perm ? row_of_.p : nullptr;
    alloc_or_throw(b_, static_cast<std::size_t>(n) * nv_, "rhs");
    alloc_or_throw(du_, static_cast<std::size_t>(n) * nv_, "du");
    cuda_check(cudaMemsetAsync(du_.p, 0, du_.count * sizeof(double), stream_), "memset");
    cuda_check(cudaMemsetAsync(b_.p, 0, b_.count * sizeof(double), stream_), "memset");
    cuda_check(cudaStreamSynchronize(stream_), "setup sync");
}

// Graph distance to the no-slip walls over the face-neighbour stencil: each
// wall face seeds its owner with the owner-to-face-centroid distance, edges
// weigh the centroid distance.  Dijkstra returns the fixed point that the
// reference's Gauss-Seidel relaxation converges to
// (MeshAuxGeometry::add_wall_distance, src/mesh/aux_geometry.cpp:609-696,
// relax_distance_graph :545-604); cells with no path keep 1e30 as there.
static std::vector<double> graph_wall_distance(const HostMesh& hm, const Csr& c2c,
                                               const std::vector<BcPatch>& patches) {
    const int32_t n = hm.n_cells;
    std::vector<double> d(static_cast<std::size_t>(n), 1.0e30);
    for (int32_t f = hm.n_inner; f < hm.n_faces; ++f) {
        if (patches[hm.patch[f]].sa_kind != 0) continue;
        const int32_t c = hm.owner[f];
        const double ex = hm.fcx[f] - hm.ccx[c], ey = hm.fcy[f] - hm.ccy[c], ez = hm.fcz[f] - hm.ccz[c];
        d[c] = std::min(d[c], std::sqrt(ex * ex + ey * ey + ez * ez));
    }
    using Item = std::pair<double, int32_t>;
    std::priority_queue<Item, std::vector<Item>, std::greater<Item>> heap;
    for (int32_t c = 0; c < n; ++c)
        if (d[c] < 1.0e30) heap.emplace(d[c], c);
    std::vector<uint8_t> done(static_cast<std::size_t>(n), 0);
    while (!heap.empty()) {
        const auto [du, u] = heap.top();
        heap.pop();
        if (done[u] || du > d[u]) continue;
        done[u] = 1;
        for (int32_t k = c2c.off[u]; k < c2c.off[u + 1]; ++k) {
            const int32_t v = c2c.val[k];
            if (done[v]) continue;
            const double dx = hm.ccx[u] - hm.ccx[v], dy = hm.ccy[u] - hm.ccy[v], dz = hm.ccz[u] - hm.ccz[v];
            const double cand = du + std::sqrt(dx * dx + dy * dy + dz * dz);
            if (cand < d[v]) {
                d[v] = cand;
                heap.emplace(cand, v);
            }
        }
    }
    return d;
}

// SpalartAllmaras::initialize (turbulence/spalart_allmaras.hpp:180-200):
// model constants, freestream nu_tilde = ratio * mu(T_inf) / rho_inf, wall
// distance, and the turbulence work arrays.
void Solver::setup_sa(const HostMesh& hm) {
    sap_.sigma = 2.0 / 3.0;
    sap_.cb1 = 0.1355;
    sap_.cb2 = 0.622;
    sap_.kappa = 0.41;
    sap_.cw2 = 0.3;
    sap_.cw3 = 2.0;
    sap_.cv1 = 7.1;
    sap_.cw1 = sap_.cb1 / (sap_.kappa * sap_.kappa) + (1.0 + sap_.cb2) / sap_.sigma;
    const double T_inf = cfg_.init_p / (cfg_.init_rho * gas_.R);
    constexpr double mu_ref = 1.716e-5, T_ref = 273.15, S_suth = 110.4;
    const double mu_inf = mu_ref * std::pow(T_inf / T_ref, 1.5) * (T_ref + S_suth) / (T_inf + S_suth);
    sap_.nu_inf = cfg_.nu_inf_ratio * mu_inf / cfg_.init_rho;
    const Csr c2c = build_cell_cells_face(hm);
    const std::vector<double> wd = graph_wall_distance(hm, c2c, patches_h_);
    upload_or_throw(wall_dist_, wd, stream_, "wall distance");
    const std::size_t n = static_cast<std::size_t>(dm_.n), nt = static_cast<std::size_t>(dm_.nt);
    const std::size_t nf = static_cast<std::size_t>(dm_.nf), nb = static_cast<std::size_t>(std::max(dm_.nb, 1));
    alloc_or_throw(rho_, nt, "rho");
    alloc_or_throw(mut_, nt, "mu_t");
    alloc_or_throw(rhonu_g_, nb, "ghost rho nu_tilde");
    alloc_or_throw(sa_face_, 2 * nf, "SA face");
    alloc_or_throw(sa_jac_, 2 * nf, "SA face jacobian");
    alloc_or_throw(sa_dsrc_, n, "SA destruction derivative");
    for (DevArray<double>* a : {&rho_, &mut_, &rhonu_g_, &sa_face_, &sa_jac_, &sa_dsrc_})
        cuda_check(cudaMemsetAsync(a->p, 0, a->count * sizeof(double), stream_), "memset");
    cuda_check(cudaStreamSynchronize(stream_), "setup sync");
    dm_.wall_dist = wall_dist_.p;
    df_.nu = q_.p + 5 * nt;  // the sixth plane of q: one gradient pass covers all six
    df_.rho = rho_.p;
    df_.mut = mut_.p;
    gnu_ = grad_.p + 15 * nt;  // nu_tilde gradient planes follow the 15 mean-flow planes
    ab_.sa_pre = n * (8.0 * 8 + 3 * 8.0) + double(dm_.nb) * (4 + 4 + 8 + 8 * 3 + 8 * 3);
    ab_.sa_grad = n * 8.0 + n * 3 * 8.0;  // nu_tilde and its three planes (stencil counted with the mean flow)
    ab_.sa_face = double(nf) * (4 * 2 + 8 * 5 + 8 * 4 + 8 * 4) + double(dm_.nb) * (4 + 8) + nt * (8 * 2 + 8 * 3 + 8);
    ab_.jac += double(nf) * 2 * 8.0 + n * 8.0;  // the face and destruction derivatives read by the 6x6 blocks
}

void Solver::sizes(int64_t* out) const {
    out[0] = dm_.n;
    out[1] = dm_.nf;
    out[2] = dm_.ni;
    out[3] = dm_.nt;
    out[4] = sys_->nnzb();
    out[5] = sys_->bs();
    out[6] = nv_;
}

// Solver::init_fields (solver.hpp:507-544): primitives_rhop_to_conserved of
// the [initial] state on every cell.
void Solver::init_fields() {
    have_prev_ = false;
    const double rho = cfg_.init_rho, p = cfg_.init_p;
    const double u = cfg_.init_velocity[0], v = cfg_.init_velocity[1], w = cfg_.init_velocity[2];
    const double T = p / (rho * gas_.R);
    const double e = gas_.cv * T;
    const double ke = 0.5 * rho * (u * u + v * v + w * w);
    const double U[5] = {rho, rho * u, rho * v, rho * w, rho * e + ke};
    for (int v5 = 0; v5 < 5; ++v5) {
        ProfScope ps(&prof_, CFDG_KCAT_UPDATE, stream_, 1, 8.0 * dm_.n);
        launch_fill(U_.p + static_cast<std::size_t>(v5) * dm_.n, dm_.n, U[v5], stream_);
    }
    if (sa_) {  // rho * nu_tilde_inf (SpalartAllmaras::initialize, spalart_allmaras.hpp:197-198)
        ProfScope ps(&prof_, CFDG_KCAT_UPDATE, stream_, 1, 8.0 * dm_.n);
        launch_fill(U_.p + static_cast<std::size_t>(5) * dm_.n, dm_.n, rho * sap_.nu_inf, stream_);
    }
    cuda_check(cudaGetLastError(), "init launch");
    if (unsteady_) reset_time_levels();  // Solver::init_fields fills U^n and U^{n-1} too (solver.hpp:525-537)
    cuda_check(cudaStreamSynchronize(stream_), "init sync");
}

void Solver::reset_time_levels() {
    if (!unsteady_) throw Failure{CFDG_ERR_INVALID, "the solver is not in unsteady mode"};
    const std::size_t bytes = U_.count * sizeof(double);
    if (!Un_.p) alloc_or_throw(Un_, U_.count, "U^n");
    if (!Unm1_.p) alloc_or_throw(Unm1_, U_.count, "U^n-1");
    cuda_check(cudaMemcpyAsync(Un_.p, U_.p, bytes, cudaMemcpyDeviceToDevice, stream_), "D2D");
    cuda_check(cudaMemcpyAsync(Unm1_.p, U_.p, bytes, cudaMemcpyDeviceToDevice, stream_), "D2D");
    cuda_check(cudaStreamSynchronize(stream_), "time levels sync");
}

void Solver::set_limiter(const double* phi, int64_t count) {
    if (!muscl_) throw Failure{CFDG_ERR_INVALID, "no limiter: the reconstruction is first order"};
    if (count < int64_t(dm_.n) * 5) throw Failure{CFDG_ERR_INVALID, "limiter array smaller than 5 x n_cells"};
    cuda_check(cudaMemcpyAsync(phi_.p, phi, sizeof(double) * 5 * dm_.n, cudaMemcpyHostToDevice, stream_), "H2D");
    cuda_check(cudaStreamSynchronize(stream_), "sync");
    limiter_frozen_ = true;
}

void Solver::set_state_host(const double* u, int64_t ld) {
    if (ld < dm_.n) throw Failure{CFDG_ERR_INVALID, "leading dimension smaller than n_cells"};
    have_prev_ = false;
    for (int v = 0; v < nv_; ++v)
        cuda_check(cudaMemcpyAsync(U_.p + static_cast<std::size_t>(v) * dm_.n, u + v * ld, sizeof(double) * dm_.n,
                                   cudaMemcpyHostToDevice, stream_),
                   "H2D");
    cuda_check(cudaStreamSynchronize(stream_), "sync");
}

void Solver::get_field(int field, double* out, int64_t count) {
    const double* src = nullptr;
    int64_t need = 0;
    const int64_t n = dm_.n, nt = dm_.nt;
    switch (field) {
        case CFDG_FIELD_U: src = U_.p; need = n * nv_; break;
        case CFDG_FIELD_Q: src = q_.p; need = nt * 5; break;
        case CFDG_FIELD_GRAD: src = grad_.p; need = need_grad_ ? nt * 3 * (sa_ ? 6 : 5) : 0; break;
        case CFDG_FIELD_PHI: src = phi_.p; need = muscl_ ? n * 5 : 0; break;
        case CFDG_FIELD_RES: src = res_.p; need = n * nv_; break;
        case CFDG_FIELD_LAM: src = lam_.p; need = n; break;
        case CFDG_FIELD_DT: src = dt_.p; need = n; break;
        case CFDG_FIELD_ALPHA: src = alpha_.p; need = n; break;
        case CFDG_FIELD_DU: src = du_.p; need = n * nv_; break;
        case CFDG_FIELD_RHS: src = b_.p; need = n * nv_; break;
        case CFDG_FIELD_MUT: src = mut_.p; need = sa_ ? nt : 0; break;
        case CFDG_FIELD_WALLDIST: src = wall_dist_.p; need = sa_ ? n : 0; break;
        case CFDG_FIELD_NU: src = df_.nu; need = sa_ ? n : 0; break;
        case CFDG_FIELD_NU_GRAD: src = gnu_; need = sa_ ? nt * 3 : 0; break;
        case CFDG_FIELD_JAC: {
            need = sys_->nnzb() * sys_->bs() * sys_->bs();
            if (count < need) throw Failure{CFDG_ERR_INVALID, "output buffer too small"};
            if (row_of_h_.empty()) {
                sys_->get_values_host(out);
                return;
            }
            // colour-ordered storage -> the reference's cell-ordered BSR
            std::vector<double> tmp(static_cast<std::size_t>(need));
            sys_->get_values_host(tmp.data());
            const auto& rp = sys_->row_ptr_host();
            const auto& cl = sys_->cols_host();
            const int64_t b2 = int64_t(sys_->bs()) * sys_->bs();
            std::vector<std::pair<int32_t, int32_t>> row;
            int64_t w = 0;
            for (int32_t c = 0; c < dm_.n; ++c) {
                const int32_t r = row_of_h_[c];
                row.clear();
                for (int32_t k = rp[r]; k < rp[r + 1]; ++k) row.emplace_back(cell_of_h_[cl[k]], k);
                std::sort(row.begin(), row.end());
                for (const auto& e : row) {
                    std::copy(tmp.begin() + e.second * b2, tmp.begin() + (e.second + 1) * b2, out + w * b2);
                    ++w;
                }
            }
            return;
        }
        default: throw Failure{CFDG_ERR_INVALID, "unknown field id"};
    }
    if (need == 0 || !src) throw Failure{CFDG_ERR_INVALID, "field not allocated for this configuration"};
    if (count < need) throw Failure{CFDG_ERR_INVALID, "output buffer too small"};
    cuda_check(cudaMemcpyAsync(out, src, sizeof(double) * need, cudaMemcpyDeviceToHost, stream_), "D2H");
    cuda_check(cudaStreamSynchronize(stream_), "sync");
    if ((field == CFDG_FIELD_DU || field == CFDG_FIELD_RHS) && !row_of_h_.empty()) {
        // linear-system vectors are stored in row (colour) order
        std::vector<double> tmp(out, out + need);
        for (int32_t c = 0; c < dm_.n; ++c)
            for (int v = 0; v < nv_; ++v) out[int64_t(c) * nv_ + v] = tmp[int64_t(row_of_h_[c]) * nv_ + v];
    }
}

void Solver::stage(int st) {
    switch (st) {
        case CFDG_STAGE_PRIMITIVES: {
            {
                ProfScope ps(&prof_, CFDG_KCAT_PRIMITIVES, stream_, 1, ab_.prim);
                launch_primitives(dm_, df_, gas_, stream_);
            }
            if (sa_) {
                ProfScope ps(&prof_, CFDG_KCAT_TURBULENCE, stream_, 1, ab_.sa_pre);
                launch_sa_pre(dm_, df_, gas_, sap_, rhonu_g_.p, stream_);
            }
            break;
        }
        case CFDG_STAGE_GRADIENT:
            if (need_grad_) {
                ProfScope ps(&prof_, CFDG_KCAT_GRADIENT, stream_, 1, ab_.grad + (sa_ ? ab_.sa_grad : 0.0));
                launch_gradient(dm_, q_.p, grad_.p, sa_ ? 6 : 5, stream_);
            }
            break;
        case CFDG_STAGE_LIMITER:
            if (need_grad_) {
                ProfScope ps(&prof_, CFDG_KCAT_LIMITER, stream_, 1,
                             muscl_ && !limiter_frozen_ ? ab_.limiter : ab_.ghost_grad);
                launch_limiter_ghostgrad(dm_, df_, gas_, muscl_ && !limiter_frozen_, cfg_.limiter, cfg_.venkat_k,
                                         stream_);
            }
            break;
        case CFDG_STAGE_FLUXES: {
            {
                ProfScope ps(&prof_, CFDG_KCAT_FACE_FLUX, stream_, 1, ab_.face_flux);
                launch_face_flux(dm_, df_, gas_, muscl_, cfg_.viscous != 0, stream_);
            }
            {
                ProfScope ps(&prof_, CFDG_KCAT_CELL_GATHER, stream_, 1, ab_.cell_gather);
                launch_cell_residual(dm_, df_, stream_);
            }
            if (sa_) {
                ProfScope ps(&prof_, CFDG_KCAT_TURBULENCE, stream_, 2, ab_.sa_face);
                launch_sa_sweep(dm_, df_, gas_, sap_, rhonu_g_.p, gnu_, sa_face_.p, sa_jac_.p, sa_dsrc_.p, stream_);
            }
            if (unsteady_) {  // step 9: the BDF pseudo-source (solver.hpp:242-246, 546-580)
                const double idt = 1.0 / cfg_.dt_physical;
                const bool bdf2 = bdf_cur_ == 2;
                const double n = double(dm_.n) * nv_;
                ProfScope ps(&prof_, CFDG_KCAT_UPDATE, stream_, 1, n * 8.0 * (bdf2 ? 5.0 : 4.0) + dm_.n * 8.0);
                launch_unsteady_source(dm_.n, nv_, vol_.p, df_.U, Un_.p, bdf2 ? Unm1_.p : nullptr,
                                       (bdf2 ? 1.5 : 1.0) * idt, (bdf2 ? -2.0 : -1.0) * idt, bdf2 ? 0.5 * idt : 0.0,
                                       df_.res, stream_);
            }
            break;
        }
        default: throw Failure{CFDG_ERR_INVALID, "unknown stage"};
    }
    cuda_check(cudaGetLastError(), "stage launch");
}

void Solver::evaluate_residual() {
    stage(CFDG_STAGE_PRIMITIVES);
    stage(CFDG_STAGE_GRADIENT);
    stage(CFDG_STAGE_LIMITER);
    stage(CFDG_STAGE_FLUXES);
}

void Solver::compute_dt(double cfl) {
    if (!(cfl > 0.0)) throw Failure{CFDG_ERR_INVALID, "CFL must be positive"};
    cfl_now_ = cfl;
    ProfScope ps(&prof_, CFDG_KCAT_UPDATE, stream_, 1, ab_.dt_rhs);
    // implicit diagonal V/dt_pseudo, plus V c0/dt of the BDF term when unsteady (solver.hpp:267-277)
    const double diag = unsteady_ ? (bdf_cur_ == 2 ? 1.5 : 1.0) / cfg_.dt_physical : 0.0;
    launch_dt_rhs(dm_, df_, nv_, cfl, diag, b_.p, stream_);
    cuda_check(cudaGetLastError(), "dt launch");
}

void Solver::assemble_jacobian() {
    JacStructure js{};
    const BsrView v = sys_->view();
    js.row_ptr = v.row_ptr;
    js.cols = v.cols;
    js.diag = v.diag;
    js.face_pos = face_pos_.p;
    js.full_viscous = cfg_.jacobian == CFDG_JAC_THIN_LAYER;
    js.sa_jac = sa_ ? sa_jac_.p : nullptr;
    js.sa_dsrc = sa_ ? sa_dsrc_.p : nullptr;
    js.cell_of = row_of_h_.empty() ? nullptr : cell_of_.p;
    {
        ProfScope ps(&prof_, CFDG_KCAT_JACOBIAN, stream_, 1,
                     ab_.jac + ab_.jac_blocks * (sys_->precision() == CFDG_PREC_MIXED ? 4.0 : 8.0));
        if (sys_->precision() == CFDG_PREC_MIXED)
            launch_jacobian<float>(dm_, df_, gas_, js, nv_, cfg_.viscous != 0, sys_->values32(), stream_);
        else
            launch_jacobian<double>(dm_, df_, gas_, js, nv_, cfg_.viscous != 0, sys_->values64(), stream_);
    }
    cuda_check(cudaGetLastError(), "jacobian launch");
}

cfdg_krylov_result Solver::linear_solve() {
    if (cfg_.precond == CFDG_PC_SGS) sys_->sgs_setup(cfg_.sgs_ordering, std::max(cfg_.sgs_sweeps, 1));
    const bool prefix = pre_freeze_phase();
    if ((guess_ && !prefix) || dataset_) prepare_guess_inputs();
    // the network predicts the update relative to the previous one: no
    // guess before a previous update exists (nor before the limiter freeze
    // under CFDG_PREFREEZE_FP64)
    const bool use_guess = guess_ && have_prev_ && !prefix;
    if (use_guess) {
        ProfScope ps(&prof_, CFDG_KCAT_GUESS, stream_, 1, double(dm_.n) * (kMlpIn * 2.0 + nv_ * 8.0));
        guess_->forward(feat_.p, dm_.n, gscale_.p + 8, du_.p, stream_);
    } else {
        cuda_check(cudaMemsetAsync(du_.p, 0, du_.count * sizeof(double), stream_), "memset");
    }
    last_jf_ = last_fallback_ = false;
    last_used_guess_ = use_guess;
    if (!jf_now()) {
        last_krylov_ = sys_->bicgstab(cfg_.precond, cfg_.lin_rel_tol, cfg_.lin_abs_tol, cfg_.lin_max_iterations,
                                      du_.p, b_.p, use_guess);
        return last_krylov_;
    }
    // Jacobian-free solve, replaced by the Picard solve when it does not
    // reduce its residual
    jf_alloc();
    {
        ProfScope ps(&prof_, CFDG_KCAT_JFNK, stream_, 2, double(dm_.n) * nv_ * 8.0);
        launch_jf_rms(dm_.n, nv_, U_.p, jf_part_.p, jf_scal_.p, stream_);
    }
    sys_->set_product([this](const double* x, double* y, const DotSpec& ds, double* partials, const int* active) {
        return jf_product(x, y, ds, partials, active);
    });
    cfdg_krylov_result kr{};
    try {
        if (cfg_.jf_krylov == CFDG_JF_GMRES)
            kr = sys_->gmres(cfg_.precond, cfg_.jf_rel_tol, cfg_.lin_abs_tol, cfg_.jf_max_iterations, cfg_.jf_restart,
                             du_.p, b_.p, use_guess);
        else
            kr = sys_->bicgstab(cfg_.precond, cfg_.jf_rel_tol, cfg_.lin_abs_tol, cfg_.jf_max_iterations, du_.p, b_.p,
                                use_guess);
    } catch (...) {
        sys_->set_product(nullptr);
        throw;
    }
    sys_->set_product(nullptr);
    const double bnorm = sys_->last_bnorm();
    if (kr.status != CFDG_KRYLOV_DIVERGED && std::isfinite(kr.final_residual) &&
        kr.final_residual <= cfg_.jf_accept * bnorm) {
        last_jf_ = true;
        last_krylov_ = kr;
        return last_krylov_;
    }
    cuda_check(cudaMemsetAsync(du_.p, 0, du_.count * sizeof(double), stream_), "memset");
    cfdg_krylov_result pk = sys_->bicgstab(cfg_.precond, cfg_.lin_rel_tol, cfg_.lin_abs_tol,
                                           cfg_.lin_max_iterations, du_.p, b_.p, false);
    pk.iterations += kr.iterations;
    last_fallback_ = true;
    last_used_guess_ = false;
    last_krylov_ = pk;
    return last_krylov_;
}

void Solver::jf_alloc() {
    if (jf_U_.p) return;
    const std::size_t n = static_cast<std::size_t>(dm_.n);
    alloc_or_throw(jf_U_, n * nv_, "perturbed state");
    alloc_or_throw(jf_res_, n * nv_, "perturbed residual");
    alloc_or_throw(jf_part_, static_cast<std::size_t>(jf_partial_blocks(dm_.n)) * 6 + 8, "product partials");
    alloc_or_throw(jf_scal_, kJfScalars, "product scalars");
    cuda_check(cudaMemsetAsync(jf_scal_.p, 0, kJfScalars * sizeof(double), stream_), "memset");
    cuda_check(cudaMallocHost(reinterpret_cast<void**>(&jf_host_), sizeof(double) * 8), "cudaMallocHost");
}

// y = (V/dt) x + (R(U + eps x) - R(U)) / eps: the residual stages run on the
// perturbed state with the perturbed residual in its own buffer (R(U) stays
// in res_ and -R(U) in b_); the primitives, gradients and face fluxes are
// overwritten and recomputed at the next evaluation.
int Solver::jf_product(const double* x, double* y, const DotSpec& ds, double* partials, const int* active) {
    const double N = double(dm_.n) * nv_;
    {
        ProfScope ps(&prof_, CFDG_KCAT_JFNK, stream_, 3, N * 8.0 * 4.0 + double(dm_.n) * 4.0);
        launch_jf_eps(dm_.n, nv_, x, jf_part_.p, jf_scal_.p, cfg_.jf_eps, active, stream_);
        launch_jf_perturb(dm_, nv_, U_.p, x, jf_scal_.p, jf_U_.p, active, stream_);
    }
    const DevFields base = df_;
    df_.U = jf_U_.p;
    df_.res = jf_res_.p;
    try {
        evaluate_residual();
    } catch (...) {
        df_ = base;
        throw;
    }
    df_ = base;
    const double diag = unsteady_ ? (bdf_cur_ == 2 ? 1.5 : 1.0) / cfg_.dt_physical : 0.0;
    ProfScope ps(&prof_, CFDG_KCAT_JFNK, stream_, 1,
                 N * 8.0 * (4.0 + (ds.n == 0 ? 0.0 : ds.n == 1 ? 1.0 : 2.0)) + double(dm_.n) * (16.0 + 4.0));
    const int nb = launch_jf_combine(dm_, nv_, alpha_.p, diag, x, b_.p, jf_res_.p, jf_scal_.p, y, ds, partials,
                                     active, stream_);
    cuda_check(cudaGetLastError(), "jacobian-free product launch");
    return nb;
}

void Solver::learn_alloc() {
    if (feat_.p) return;
    const std::size_t n = static_cast<std::size_t>(dm_.n);
    alloc_or_throw(feat_, n * kMlpIn, "guess features");
    alloc_or_throw(du_prev_, n * nv_, "previous update");
    alloc_or_throw(gscale_, 32, "guess scales");
    alloc_or_throw(gpart_, static_cast<std::size_t>(guess_sum_blocks(dm_.n)) * 2 * nv_ + 8, "guess partials");
    cuda_check(cudaMemsetAsync(du_prev_.p, 0, du_prev_.count * sizeof(double), stream_), "memset");
    // free-stream scales and state (conserved) for the state features
    const double rho = cfg_.init_rho, p = cfg_.init_p;
    const double u = cfg_.init_velocity[0], v = cfg_.init_velocity[1], w = cfg_.init_velocity[2];
    const double T = p / (rho * gas_.R);
    const double a = std::sqrt(gas_.gamma * gas_.R * T);
    const double E = rho * gas_.cv * T + 0.5 * rho * (u * u + v * v + w * w);
    const double spd = std::max(std::sqrt(u * u + v * v + w * w), a);
    double h[32] = {};
    const double su[6] = {rho, rho * spd, rho * spd, rho * spd, E, sa_ ? std::max(rho * sap_.nu_inf, 1e-300) : 1.0};
    const double ui[6] = {rho, rho * u, rho * v, rho * w, E, sa_ ? rho * sap_.nu_inf : 0.0};
    for (int k = 0; k < 8; ++k) h[k] = h[8 + k] = 1.0;
    for (int k = 0; k < 6; ++k) {
        h[16 + k] = su[k];
        h[24 + k] = ui[k];
    }
    cuda_check(cudaMemcpyAsync(gscale_.p, h, sizeof(h), cudaMemcpyHostToDevice, stream_), "H2D");
    cuda_check(cudaStreamSynchronize(stream_), "sync");
}

void Solver::prepare_guess_inputs() {
    ProfScope ps(&prof_, CFDG_KCAT_GUESS, stream_, 3,
                 double(dm_.n) * (nv_ * 8.0 * 4 + 16.0) +
                     double(dm_.n) * (kMlpIn * 2.0 + 8.0 * (nv_ * 3 + 2)) + double(c2c_.count) * 4.0);
    launch_guess_scales(dm_.n, dm_.row_of, nv_, b_.p, dt_.p, vol_.p, du_prev_.p, gpart_.p, gscale_.p, stream_);
    launch_guess_features(dm_, nv_, U_.p, b_.p, dt_.p, du_prev_.p, gscale_.p, cfl_now_, feat_.p, stream_);
    cuda_check(cudaGetLastError(), "guess launch");
}

void Solver::attach_guess(Mlp* m) {
    if (m && (m->nvars() != nv_ || m->device() != device_))
        throw Failure{CFDG_ERR_INVALID, "network variable count or device does not match the solver"};
    if (m) learn_alloc();
    guess_ = m;
}

void Solver::attach_dataset(Dataset* d, int32_t stride) {
    if (d && (d->nvars() != nv_ || d->device() != device_))
        throw Failure{CFDG_ERR_INVALID, "dataset variable count or device does not match the solver"};
    if (d && stride < 1) throw Failure{CFDG_ERR_INVALID, "dataset stride must be >= 1"};
    if (d) learn_alloc();
    dataset_ = d;
    ds_stride_ = std::max(stride, 1);
    ds_phase_ = 0;
}

void Solver::residual_norms(double* l2_host) {
    {
        ProfScope ps(&prof_, CFDG_KCAT_UPDATE, stream_, 2, ab_.norms);
        launch_norms(dm_.n, nv_, res_.p, norm_partials_.p, l2_.p, stream_);
    }
    cuda_check(cudaMemcpyAsync(l2_host_, l2_.p, sizeof(double) * nv_, cudaMemcpyDeviceToHost, stream_), "D2H");
    cuda_check(cudaStreamSynchronize(stream_), "norm sync");
    prof_.collect();
    for (int v = 0; v < nv_; ++v) l2_host[v] = l2_host_[v];
}

cfdg_step_result Solver::newton_step(double cfl) {
    cfdg_step_result r{};
    sys_->set_precision(pre_freeze_phase() ? CFDG_PREC_FP64 : cfg_.precision);
    evaluate_residual();
    compute_dt(cfl);
    assemble_jacobian();
    const cfdg_krylov_result kr = linear_solve();
    if (dataset_ && have_prev_) {
        const int64_t want = (int64_t(dm_.n) - ds_phase_ + ds_stride_ - 1) / ds_stride_;
        const int64_t at = dataset_->size();
        const int64_t got = dataset_->reserve(want);
        if (got > 0) {
            ProfScope ps(&prof_, CFDG_KCAT_GUESS, stream_, 1, double(got) * (kMlpIn * 4.0 + nv_ * 8.0 + kMlpOut * 4.0));
            launch_guess_append(dm_.n, dm_.row_of, nv_, ds_stride_, ds_phase_, got, feat_.p, du_.p, gscale_.p,
                                dataset_->X() + at * kMlpIn, dataset_->T() + at * kMlpOut, stream_);
        }
        ds_phase_ = (ds_phase_ + 1) % ds_stride_;
    }
    const double* scale = nullptr;
    if (last_jf_ && cfg_.jf_max_change > 0.0) {
        ProfScope ps(&prof_, CFDG_KCAT_JFNK, stream_, 2, double(dm_.n) * (nv_ * 8.0 + 16.0 + 4.0));
        launch_jf_step_scale(dm_, nv_, U_.p, du_.p, jf_part_.p, jf_scal_.p, cfg_.jf_max_change, stream_);
        scale = jf_scal_.p + kJfStep;
        cuda_check(cudaMemcpyAsync(jf_host_, scale, sizeof(double), cudaMemcpyDeviceToHost, stream_), "D2H");
    }
    {
        ProfScope ps(&prof_, CFDG_KCAT_UPDATE, stream_, 1, ab_.state_update);
        launch_state_update(dm_, U_.p, du_.p, nv_, scale, stream_);
    }
    if (guess_ || dataset_) {
        cuda_check(cudaMemcpyAsync(du_prev_.p, du_.p, du_.count * sizeof(double), cudaMemcpyDeviceToDevice, stream_),
                   "D2D");
        have_prev_ = true;
    }
    residual_norms(r.l2);  // synchronises the stream: jf_host_ is valid after it
    r.cfl = cfl;
    r.nvars = nv_;
    r.jacobian_free = last_jf_ ? 1 : 0;
    r.picard_fallback = last_fallback_ ? 1 : 0;
    r.step_scale = scale ? jf_host_[0] : 1.0;
    r.krylov_status = kr.status;
    r.krylov_iterations = kr.iterations;
    r.krylov_initial = kr.initial_residual;
    r.krylov_final = kr.final_residual;
    r.guess_used = last_used_guess_ ? sys_->last_guess() : 0;
    r.krylov_rhs = sys_->last_bnorm();
    return r;
}

// Geometric CFL ramp from cfl to cfl_max over cfl_ramp_iterations
// iterations (the reference holds CFL constant, solver.hpp:265).
double Solver::cfl_at(int64_t iter) const {
    const int K = cfg_.cfl_ramp_iterations;
    if (K <= 1 || !(cfg_.cfl_max > cfg_.cfl)) return cfg_.cfl;
    const double t = std::min(1.0, double(iter - 1) / double(K - 1));
    return std::min(cfg_.cfl_max, cfg_.cfl * std::pow(cfg_.cfl_max / cfg_.cfl, t));
}

// Solver::run_steady (solver.hpp:597-660) with the CFL ramp and the
// selected convergence monitor.
cfdg_run_result Solver::run_steady() {
    cfdg_run_result out{};
    const auto t0 = std::chrono::steady_clock::now();
    double ref_norm[6] = {0, 0, 0, 0, 0, 0};
    bool have0 = false;
    const int interval = std::max(cfg_.residual_interval, 1);
    const bool robust = cfg_.convergence_monitor == 1;
    // switched evolution relaxation: the monitor at the ramp's end
    const bool ser = cfg_.cfl_ser_max > cfg_.cfl_max;
    const int64_t ramp = std::max(cfg_.cfl_ramp_iterations, 1);
    double rel_ramp = -1.0;
    for (int64_t iter = 1; iter <= cfg_.max_iterations; ++iter) {
        cfdg_step_result st;
        if (cfg_.limiter_freeze > 0 && iter >= cfg_.limiter_freeze) limiter_frozen_ = true;
        double cfl = cfl_at(iter);
        if (ser && rel_ramp > 0.0 && iter > ramp && out.rel > 0.0)
            cfl = std::min(cfg_.cfl_ser_max, cfg_.cfl_max * std::max(1.0, rel_ramp / out.rel));
        out.cfl_last = cfl;
        try {
            st = newton_step(cfl);
        } catch (const Failure& f) {
            // a non-finite state shows up in the diagonal blocks before the
            // residual norms: the reference's "blowup" exit (solver.hpp:625-629)
            if (f.status != CFDG_ERR_NONFINITE) throw;
            out.iterations = iter;
            out.blowup = 1;
            break;
        }
        out.iterations = iter;
        out.krylov_iterations_total += st.krylov_iterations;
        out.jacobian_free_steps += st.jacobian_free;
        out.picard_fallbacks += st.picard_fallback;
        const bool diagnose = iter == 1 || iter % interval == 0 || iter == cfg_.max_iterations;
        if (!diagnose) continue;
        bool finite = true;
        for (int v = 0; v < nv_; ++v) finite = finite && std::isfinite(st.l2[v]);
        if (!finite) {
            out.blowup = 1;
            break;
        }
        for (int v = 0; v < nv_; ++v) out.l2_last[v] = st.l2[v];
        // monitored components
        double mon[6];
        int nm = 0;
        if (robust) {
            mon[nm++] = st.l2[0];
            mon[nm++] = std::sqrt(st.l2[1] * st.l2[1] + st.l2[2] * st.l2[2] + st.l2[3] * st.l2[3]);
            mon[nm++] = st.l2[4];
            if (nv_ == 6) mon[nm++] = st.l2[5];
        } else {
            for (int v = 0; v < nv_; ++v) mon[nm++] = st.l2[v];
        }
        if (!have0) {
            for (int v = 0; v < nv_; ++v) out.l2_first[v] = st.l2[v];
            for (int k = 0; k < nm; ++k) ref_norm[k] = mon[k];
            have0 = true;
            out.rel = 1.0;
            continue;
        }
        if (robust)
            for (int k = 0; k < nm; ++k) ref_norm[k] = std::max(ref_norm[k], mon[k]);
        double rel = 0.0;
        for (int k = 0; k < nm; ++k) rel = std::max(rel, mon[k] / std::max(ref_norm[k], 1.0e-300));
        out.rel = rel;
        if (ser && rel_ramp < 0.0 && iter >= ramp) rel_ramp = rel;
        if (rel <= cfg_.residual_tolerance) {
            out.converged = 1;
            break;
        }
    }
    out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return out;
}

// Solver::run_dual_time (solver.hpp:662-736): per physical step BDF1 on the
// first and BDF order afterwards, Newton sub-iterations until the monitor
// (sub-iteration 1, every 5th and the last) drops below the tolerance, then
// U^{n-1} <- U^n, U^n <- U (shift_physical_time_levels, solver.hpp:582-596).
cfdg_unsteady_result Solver::run_unsteady() {
    if (!unsteady_) throw Failure{CFDG_ERR_INVALID, "cfdg_run_unsteady: time_mode is not CFDG_TIME_UNSTEADY"};
    if (!Un_.p) reset_time_levels();
    cfdg_unsteady_result out{};
    const auto t0 = std::chrono::steady_clock::now();
    const bool robust = cfg_.convergence_monitor == 1;
    const std::size_t bytes = U_.count * sizeof(double);
    for (int64_t step = 1; step <= cfg_.max_time_steps; ++step) {
        bdf_cur_ = (step == 1 || cfg_.bdf_order == 1) ? 1 : 2;
        double ref_norm[6] = {0, 0, 0, 0, 0, 0};
        bool have0 = false, converged = false;
        for (int64_t sub = 1; sub <= cfg_.max_iterations; ++sub) {
            cfdg_step_result st;
            try {
                st = newton_step(cfl_at(sub));
            } catch (const Failure& f) {
                if (f.status != CFDG_ERR_NONFINITE) throw;
                out.blowup = 1;
                break;
            }
            ++out.subiterations_total;
            out.krylov_iterations_total += st.krylov_iterations;
            for (int v = 0; v < nv_; ++v) out.l2_last[v] = st.l2[v];
            const bool diagnose = sub == 1 || sub % 5 == 0 || sub == cfg_.max_iterations;
            if (!diagnose) continue;
            bool finite = true;
            for (int v = 0; v < nv_; ++v) finite = finite && std::isfinite(st.l2[v]);
            if (!finite) {
                out.blowup = 1;
                break;
            }
            double mon[6];
            int nm = 0;
            if (robust) {
                mon[nm++] = st.l2[0];
                mon[nm++] = std::sqrt(st.l2[1] * st.l2[1] + st.l2[2] * st.l2[2] + st.l2[3] * st.l2[3]);
                mon[nm++] = st.l2[4];
                if (nv_ == 6) mon[nm++] = st.l2[5];
            } else {
                for (int v = 0; v < nv_; ++v) mon[nm++] = st.l2[v];
            }
            if (!have0) {
                for (int k = 0; k < nm; ++k) ref_norm[k] = mon[k];
                have0 = true;
                continue;
            }
            double rel = 0.0;
            for (int k = 0; k < nm; ++k) {
                if (robust) ref_norm[k] = std::max(ref_norm[k], mon[k]);
                rel = std::max(rel, mon[k] / std::max(ref_norm[k], 1.0e-300));
            }
            if (rel <= cfg_.residual_tolerance) {
                converged = true;
                break;
            }
        }
        if (out.blowup) break;
        out.time_steps = step;
        out.t_physical = double(step) * cfg_.dt_physical;
        if (converged) ++out.steps_converged;
        // U^{n-1} <- U^n, U^n <- U
        std::swap(Un_.p, Unm1_.p);
        cuda_check(cudaMemcpyAsync(Un_.p, U_.p, bytes, cudaMemcpyDeviceToDevice, stream_), "D2D");
    }
    cuda_check(cudaStreamSynchronize(stream_), "unsteady sync");
    out.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return out;
}

}  // namespace cfdg
