// Host-side objects behind the C ABI: the block-sparse linear system
// (BsrMatrix + SgsPreconditioner + BiCGSTAB of the reference linalg module)
// and the compressible solver (Solver<...> + BackwardEuler).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "cfdg.h"
#include "device_common.cuh"
#include "host_mesh.hpp"
#include "kernels.hpp"
#include "guess.hpp"
#include "krylov.hpp"

namespace cfdg {

void set_error(const std::string& msg);

// Least-squares gradient coefficients in warp slices (DevMesh::g_soff):
// slot offsets per slice, neighbour per slot, coefficients per slot, and
// the stencil's entry count before padding.
struct LsqSlices {
    std::vector<int64_t> soff;
    std::vector<int32_t> col;
    std::vector<double> wx, wy, wz;
    int64_t entries = 0;
};
LsqSlices build_lsq_slices(const HostMesh& hm, const Csr& st);

// Owning device allocation.
template <typename T>
struct DevArray {
    T* p = nullptr;
    std::size_t count = 0;
    DevArray() = default;
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    ~DevArray() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        count = 0;
    }
    bool alloc(std::size_t n) {
        release();
        if (n == 0) return true;
        if (cudaMalloc(reinterpret_cast<void**>(&p), n * sizeof(T)) != cudaSuccess) {
            p = nullptr;
            return false;
        }
        count = n;
        return true;
    }
    bool upload(const T* h, std::size_t n, cudaStream_t s) {
        if (!alloc(n)) return false;
        if (n == 0) return true;
        return cudaMemcpyAsync(p, h, n * sizeof(T), cudaMemcpyHostToDevice, s) == cudaSuccess;
    }
    bool upload(const std::vector<T>& h, cudaStream_t s) { return upload(h.data(), h.size(), s); }
};

// Thrown inside the library; converted to a status code at the C boundary.
struct Failure {
    int status;
    std::string msg;
};

template <typename T>
void upload_or_throw(DevArray<T>& a, const std::vector<T>& h, cudaStream_t s, const char* what) {
    if (!a.upload(h, s)) throw Failure{CFDG_ERR_NOMEM, std::string("device allocation failed: ") + what};
}
template <typename T>
void alloc_or_throw(DevArray<T>& a, std::size_t n, const char* what) {
    if (!a.alloc(n)) throw Failure{CFDG_ERR_NOMEM, std::string("device allocation failed: ") + what};
}
void cuda_check(cudaError_t e, const char* what);

// Optional per-launch timing with CUDA events recorded on the launching
// stream; launch counting is always on.
class Profiler {
public:
    ~Profiler();
    void enable(bool on);
    bool on() const { return on_; }
    void start(int cat, cudaStream_t s);
    void stop(cudaStream_t s);
    void collect();  // resolves recorded pairs; the stream must be idle
    void add_bytes(int cat, double b) {
        if (on_) bytes[cat] += b;
    }
    double ms[CFDG_KCAT_COUNT] = {};
    int64_t count[CFDG_KCAT_COUNT] = {};
    double bytes[CFDG_KCAT_COUNT] = {};  // algorithmic (unique-touch) bytes of the timed launches
    int64_t launches = 0;

private:
    cudaEvent_t get();
    struct Rec {
        int cat;
        cudaEvent_t a, b;
    };
    bool on_ = false;
    std::vector<cudaEvent_t> free_, all_;
    std::vector<Rec> pending_;
    int open_cat_ = -1;
    cudaEvent_t open_ = nullptr;
};

struct ProfScope {
    Profiler* p;
    cudaStream_t s;
    ProfScope(Profiler* prof, int cat, cudaStream_t st, int n = 1, double bytes = 0.0) : p(prof), s(st) {
        p->launches += n;
        if (p->on()) {
            p->bytes[cat] += bytes;
            p->start(cat, s);
        }
    }
    ~ProfScope() {
        if (p->on()) p->stop(s);
    }
};

// Block-sparse matrix with its SGS preconditioner and BiCGSTAB workspace.
class BsrSystem {
public:
    BsrSystem(int device, int32_t n, int32_t bs, const int32_t* row_ptr, const int32_t* cols, int precision,
              cudaStream_t stream);
    ~BsrSystem();

    int32_t n() const { return n_; }
    int32_t bs() const { return bs_; }
    int64_t nnzb() const { return nnzb_; }
    int precision() const { return precision_; }
    cudaStream_t stream() const { return stream_; }
    BsrView view() const { return BsrView{n_, bs_, row_ptr_.p, cols_.p, diag_.p}; }
    const int32_t* diag_host() const { return diag_h_.data(); }
    const std::vector<int32_t>& row_ptr_host() const { return row_ptr_h_; }
    const std::vector<int32_t>& cols_host() const { return cols_h_; }
    double* values64() { return vals64_.p; }
    float* values32() { return vals32_.p; }

    // Switches the stored matrix precision (CFDG_PREC_*): values and block
    // LU of the new precision are allocated, the other precision's released,
    // and set-up must run again before the next apply.
    void set_precision(int precision);
    void set_values_host(const double* v);
    void get_values_host(double* v);
    // y = alpha*A*x + beta*y (device vectors)
    void spmv(const double* x, double* y, double alpha, double beta);
    // SgsPreconditioner::setup: ordering + block LU of the diagonal.
    void sgs_setup(int ordering, int sweeps);
    // z = M^-1 r (device vectors).
    void sgs_apply(const double* r, double* z, const int* active);
    // z = M^-1 r, then y = A z with the dots `ds` (partials at `partials`);
    // with the split multicolour sweep the product on colour 0 is fused into
    // its last pass.  Returns the number of partial rows written.
    int sgs_apply_spmv(const double* r, double* z, double* y, const DotSpec& ds, double* partials, const int* active);
    // BiCGSTAB on device vectors; x holds the initial guess.
    // guess: x holds an initial guess that is replaced by x = 0 when
    // ||b - A x|| >= ||b||; last_guess() tells 1 accepted, 2 rejected.
    cfdg_krylov_result bicgstab(int precond, double rel_tol, double abs_tol, int max_it, double* x, const double* b,
                                bool guess = false);
    // Restarted GMRES(restart), right-preconditioned, on the same operator
    // (the stored matrix or the matrix-free product); same conventions as
    // bicgstab.  The basis is allocated on first use.
    cfdg_krylov_result gmres(int precond, double rel_tol, double abs_tol, int max_it, int restart, double* x,
                             const double* b, bool guess = false);
    int last_guess() const { return last_guess_; }
    double last_bnorm() const { return last_bnorm_; }
    int groups_fwd() const { return static_cast<int>(fwd_off_.size()) - 1; }
    int groups_bwd() const { return static_cast<int>(bwd_off_.size()) - 1; }
    int64_t launches() const { return prof_->launches; }
    void set_profiler(Profiler* p) { prof_ = p ? p : &own_prof_; }
    Profiler* profiler() { return prof_; }
    // Matrix-free Krylov operator: y = Op x with the dots `ds`, returning
    // the partial rows written (null: the stored matrix).  The preconditioner
    // keeps using the stored matrix; the iterations run in the host loop.
    using Product = std::function<int(const double* x, double* y, const DotSpec& ds, double* partials,
                                      const int* active)>;
    void set_product(Product p) { product_ = std::move(p); }
    int check_every = 1;  // host loop: polls the Krylov state every k iterations
    bool device_loop = true;  // run the iterations as one graph launch (CFDG_KRYLOV_DEVICE_LOOP)

private:
    void build_ordering(int ordering);
    template <typename F>
    bool device_loop_ready(int precond, double* x, const double* b, F&& iteration);
    void release_device_loop();
    template <typename MT>
    void sgs_apply_t(const MT* vals, const MT* lu, const double* r, double* z, const int* active,
                     bool skip_last = false);
    bool fuse_last_spmv() const { return split_ && sweeps_ == 1 && groups_bwd() >= 2; }

    int device_;
    cudaStream_t stream_;
    int32_t n_, bs_;
    int64_t nnzb_;
    int precision_;
    std::vector<int32_t> row_ptr_h_, cols_h_, diag_h_;
    DevArray<int32_t> row_ptr_, cols_, diag_;
    DevArray<double> vals64_, lu64_;
    DevArray<float> vals32_, lu32_;
    DevArray<int8_t> piv_;
    DevArray<int> err_;
    int ordering_ = -1, sweeps_ = 1;
    int last_guess_ = 0;
    double last_bnorm_ = 0.0;
    bool lu_ready_ = false;
    std::vector<int32_t> fwd_off_, bwd_off_;
    std::vector<int32_t> fwd_first_, bwd_first_;  // first row of a contiguous group, -1 otherwise
    // algorithmic bytes of one pass, mode 0 / 1 / split half: the part that
    // does not depend on the matrix precision, and the matrix blocks read
    std::vector<double> fwd_bytes_[3], bwd_bytes_[3], fwd_blocks_[3], bwd_blocks_[3];
    double block_bytes() const { return double(bs_) * bs_ * (precision_ == CFDG_PREC_MIXED ? 4.0 : 8.0); }
    bool split_ = false;  // colour-ordered matrix: first sweep split at the diagonal
    DevArray<int32_t> fwd_rows_, bwd_rows_;
    DevArray<int32_t> fwd_off_d_, bwd_off_d_;  // level boundaries on the device (cooperative level sweep)
    DevArray<int4> fwd_meta_, bwd_meta_;       // (row, first block, block end, diagonal) in level order
    bool level_coop_ = true;                  // cleared when the cooperative launch is unavailable
    double spmv_bytes(int n_extra_vectors, bool read_y) const;
    // rows [fwd_off_[1], n) of a colour-ordered matrix: block count and
    // distinct columns (the SpMV left after the fused colour-0 product)
    double rest_nnzb_ = 0.0, rest_cols_ = 0.0;
    // Krylov workspace
    DevArray<double> r_, r0_, p_, v_, s_, t_, phat_, shat_, partials_;
    DevArray<KrylovScalars> ks_;
    KrylovScalars* ks_host_ = nullptr;
    // device loop (graph with a conditional while-node), keyed by what the
    // captured launches read
    struct LoopKey {
        int precond = -1;
        const double* x = nullptr;
        const double* b = nullptr;
        int ordering = -1, sweeps = 0, precision = -1;
        bool operator==(const LoopKey& o) const {
            return precond == o.precond && x == o.x && b == o.b && ordering == o.ordering && sweeps == o.sweeps &&
                   precision == o.precision;
        }
    };
    LoopKey loop_key_;
    cudaGraphExec_t loop_exec_ = nullptr;
    cudaGraphConditionalHandle loop_handle_{};
    int64_t loop_body_launches_ = 0;
    bool loop_failed_ = false;
    Profiler own_prof_;
    Profiler* prof_ = &own_prof_;
    Product product_;
    // GMRES workspace: basis (restart + 1 vectors), a vector, partials,
    // device and pinned host coefficients (3 x (restart + 1) + 8)
    DevArray<double> gm_V_, gm_z_, gm_part_, gm_h_;
    double* gm_h_host_ = nullptr;
    int gm_restart_ = 0;
    void gm_alloc(int restart);
};

// The compressible finite-volume solver on one device.
class Solver {
public:
    Solver(int device, const cfdg_mesh_host& mesh, const cfdg_config& cfg, const cfdg_bc_desc* bcs, int n_bcs);
    ~Solver();

    void init_fields();
    void set_state_host(const double* u, int64_t ld);
    void get_field(int field, double* out, int64_t count);
    void evaluate_residual();
    void stage(int st);
    void compute_dt(double cfl);
    void assemble_jacobian();
    cfdg_krylov_result linear_solve();
    cfdg_step_result newton_step(double cfl);
    void residual_norms(double* l2_host);
    cfdg_run_result run_steady();
    cfdg_unsteady_result run_unsteady();
    // Solver::write_fields: <outdir>/<stem>_00000.vtu + <stem>.pvtu of the
    // current state on `mesh` (the mesh the solver was created with)
    void write_vtu(const cfdg_mesh_host& mesh, const std::string& outdir, const std::string& stem);
    void reset_time_levels();
    cudaStream_t stream() const { return stream_; }
    int64_t launches() const { return prof_.launches; }
    Profiler& profiler() { return prof_; }
    BsrSystem& system() { return *sys_; }
    void sizes(int64_t* out) const;
    double cfl_at(int64_t iter) const;
    // learned initial guess of the linear solve (nullptr: zero guess) and
    // the dataset that receives (features, dU) of every stride-th cell
    void attach_guess(Mlp* m);
    void attach_dataset(Dataset* d, int32_t stride);
    void freeze_limiter(bool frozen) { limiter_frozen_ = frozen; }
    // CFDG_PREFREEZE_FP64 and the limiter not yet frozen: FP64 matrix, zero
    // initial guess
    bool pre_freeze_phase() const { return cfg_.pre_freeze == CFDG_PREFREEZE_FP64 && !limiter_frozen_; }
    void set_limiter(const double* phi, int64_t count);

private:
    void setup_mesh(const cfdg_mesh_host& mesh);
    void setup_bcs(const cfdg_bc_desc* bcs, int n_bcs, const HostMesh& hm);
    void setup_matrix(const HostMesh& hm, const Csr& c2c);
    void setup_sa(const HostMesh& hm);
    void rhs_update_ready();

    int device_;
    cudaStream_t stream_ = nullptr;
    cfdg_config cfg_;
    GasParams gas_;
    int nv_ = 5;
    bool sa_ = false;
    bool need_grad_ = false;
    bool muscl_ = false;
    bool limiter_frozen_ = false;
    // dual time stepping: physical time levels U^n, U^{n-1} and the BDF
    // order of the current physical step
    bool unsteady_ = false;
    int bdf_cur_ = 1;
    DevArray<double> Un_, Unm1_;
    Mlp* guess_ = nullptr;
    Dataset* dataset_ = nullptr;
    int32_t ds_stride_ = 1, ds_phase_ = 0;
    DevArray<uint16_t> feat_;
    DevArray<double> du_prev_, gscale_, gpart_;
    double cfl_now_ = 1.0;
    bool have_prev_ = false, last_used_guess_ = false;
    void prepare_guess_inputs();
    void learn_alloc();
    // Jacobian-free Newton-Krylov (CFDG_NEWTON_JACOBIAN_FREE): the perturbed
    // state and its residual (SoA, cell order), reduction partials, the
    // device scalars (kJfScalars) and a pinned host copy of the step factor
    DevArray<double> jf_U_, jf_res_, jf_part_, jf_scal_;
    double* jf_host_ = nullptr;
    bool last_jf_ = false, last_fallback_ = false;
    bool jf_now() const {
        return cfg_.newton_operator == CFDG_NEWTON_JACOBIAN_FREE && (!muscl_ || limiter_frozen_);
    }
    void jf_alloc();
    int jf_product(const double* x, double* y, const DotSpec& ds, double* partials, const int* active);
    DevMesh dm_{};
    DevFields df_{};
    SaParams sap_{};
    // mesh arrays
    DevArray<int32_t> owner_, neigh_, bpatch_, c2f_off_, c2f_, c2fs_, c2c_off_, c2c_, g_col_;
    DevArray<int64_t> g_soff_;
    int64_t g_entries_ = 0;  // stencil entries before the slice padding
    DevArray<double> fnx_, fny_, fnz_, farea_, fcx_, fcy_, fcz_, fdx_, fdy_, fdz_, finv_d_, ccx_, ccy_, ccz_, vol_,
        g_wx_, g_wy_, g_wz_, wall_dist_;
    DevArray<BcPatch> patches_;
    std::vector<BcPatch> patches_h_;
    // fields
    DevArray<double> U_, q_, grad_, phi_, fflux_, res_, lam_, dt_, alpha_;
    // Spalart-Allmaras: rho, mu_t (n_total), ghost rho*nu_tilde (nb), face
    // flux + spectral increments (2 nf), face d flux / d(rho nu_tilde) (2 nf),
    // destruction derivative (n); nu_tilde is plane 5 of q_ and its gradient
    // grad_ planes 15..17
    DevArray<double> rho_, mut_, rhonu_g_, sa_face_, sa_jac_, sa_dsrc_;
    double* gnu_ = nullptr;
    // linear system
    std::unique_ptr<BsrSystem> sys_;
    DevArray<int32_t> face_pos_, row_of_, cell_of_;
    std::vector<int32_t> row_of_h_, cell_of_h_;  // colour-ordered system: cell -> row, row -> cell
    DevArray<double> b_, du_, norm_partials_, l2_;
    double* l2_host_ = nullptr;
    Profiler prof_;
    // algorithmic (unique-touch) bytes per launch of each residual-side kernel
    struct {
        double prim, grad, limiter, ghost_grad, face_flux, cell_gather, jac, jac_blocks, dt_rhs, state_update, norms;
        double sa_pre, sa_grad, sa_face;
    } ab_{};
    void compute_alg_bytes(int64_t n_grad_edges, int64_t n_c2c, int64_t n_c2f);
    cfdg_krylov_result last_krylov_{};
};

}  // namespace cfdg
