// extern "C" entry points of include/cfdg.h.  Every call converts library
// failures into a status code and keeps the message for cfdg_last_error().
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <exception>
#include <new>
#include <string>

#include "cfdg.h"
#include "halo.hpp"
#include "host_mesh.hpp"
#include "recon.hpp"
#include "solver.hpp"

struct cfdg_solver {
    cfdg::Solver* impl;
    int device;
};
struct cfdg_bsr {
    cudaStream_t stream;
    cfdg::BsrSystem* impl;
    int device;
};
struct cfdg_host_mesh {
    cfdg::HostMesh mesh;
};
struct cfdg_mlp {
    cfdg::Mlp* impl;
    cudaStream_t stream;
    int device;
};
struct cfdg_dataset {
    cfdg::Dataset* impl;
    int device;
};
struct cfdg_recon {
    cfdg::ReconOperator* impl;
};
struct cfdg_halo {
    cfdg::HaloPlan plan;
};

namespace cfdg {
namespace {
thread_local std::string g_last_error;
}
void set_error(const std::string& msg) { g_last_error = msg; }
}  // namespace cfdg

namespace {

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return CFDG_OK;
    } catch (const cfdg::Failure& e) {
        cfdg::set_error(e.msg);
        return e.status;
    } catch (const std::bad_alloc&) {
        cfdg::set_error("host allocation failed");
        return CFDG_ERR_NOMEM;
    } catch (const std::exception& e) {
        cfdg::set_error(e.what());
        return CFDG_ERR_INVALID;
    } catch (...) {
        cfdg::set_error("unknown failure");
        return CFDG_ERR_INVALID;
    }
}

int require_device(int device) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0) {
        cudaGetLastError();
        cfdg::set_error("no CUDA device visible");
        return CFDG_ERR_NODEVICE;
    }
    if (device < 0 || device >= count) {
        cfdg::set_error("device index out of range");
        return CFDG_ERR_INVALID;
    }
    return CFDG_OK;
}

}  // namespace

namespace {
// uploads the plan's index lists to `device` on first use
int halo_device_ready(cfdg_halo* h, int device, int32_t nvars) {
    if (nvars < 1 || nvars > cfdg::kHaloMaxVars) {
        cfdg::set_error("halo: nvars (or the block size) must be in [1, 32]");
        return CFDG_ERR_INVALID;
    }
    const int dv = require_device(device);
    if (dv != CFDG_OK) return dv;
    cfdg::HaloPlan& p = h->plan;
    if (p.device >= 0 && p.device != device) {
        cfdg::set_error("halo: the plan's index lists live on another device");
        return CFDG_ERR_INVALID;
    }
    return guarded([&] {
        cfdg::cuda_check(cudaSetDevice(device), "cudaSetDevice");
        if (p.device < 0) {
            cfdg::upload_or_throw(p.send_d, p.send_owned_local, nullptr, "halo send list");
            cfdg::upload_or_throw(p.recv_d, p.recv_ghost_local, nullptr, "halo recv list");
            cfdg::cuda_check(cudaStreamSynchronize(nullptr), "halo upload");
            p.device = device;
        }
    });
}
}  // namespace

extern "C" {

int cfdg_version(void) { return 10000; }

const char* cfdg_status_string(int status) {
    switch (status) {
        case CFDG_OK: return "ok";
        case CFDG_ERR_INVALID: return "invalid argument";
        case CFDG_ERR_CUDA: return "CUDA error";
        case CFDG_ERR_NOMEM: return "out of memory";
        case CFDG_ERR_SINGULAR: return "singular diagonal block";
        case CFDG_ERR_NONFINITE: return "non-finite value";
        case CFDG_ERR_DIVERGED: return "Krylov breakdown";
        case CFDG_ERR_MESH: return "invalid mesh";
        case CFDG_ERR_UNSUPPORTED: return "unsupported option";
        case CFDG_ERR_NODEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

const char* cfdg_last_error(void) { return cfdg::g_last_error.c_str(); }

int cfdg_device_count(int* count_h) {
    if (!count_h) return CFDG_ERR_INVALID;
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) {
        cudaGetLastError();
        c = 0;
    }
    *count_h = c;
    return CFDG_OK;
}

void cfdg_config_default(cfdg_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    // SolverConfig / SolverParams defaults (solver/compressible/config.hpp:94-136,
    // linalg/config.hpp:14-26), implicit MUSCL + LSQ as on the hot path.
    c->viscous = 0;
    c->turbulence = 0;
    c->gradient = CFDG_GRAD_LSQ_NODE;
    c->reconstruction = CFDG_RECON_MUSCL;
    c->limiter = CFDG_LIM_VENKATAKRISHNAN;
    c->precision = CFDG_PREC_FP64;
    c->precond = CFDG_PC_SGS;
    c->sgs_ordering = CFDG_SGS_COLOR;
    c->sgs_sweeps = 1;
    c->lin_max_iterations = 500;
    c->cfl_ramp_iterations = 0;
    c->residual_interval = 1;
    c->gamma = 1.4;
    c->gas_constant = 287.052874;
    c->prandtl = 0.71;
    c->prandtl_turb = 0.9;
    c->init_rho = 1.225;
    c->init_p = 101325.0;
    c->venkat_k = 0.5;
    c->cfl = 0.4;
    c->cfl_max = 0.4;
    c->residual_tolerance = 1.0e-10;
    c->lin_rel_tol = 1.0e-1;
    c->lin_abs_tol = 1.0e-15;
    c->nu_inf_ratio = 3.0;
    c->max_iterations = 10000;
    // SolverConfig [time] defaults (config.hpp:117-125)
    c->dt_physical = 1.0e-6;
    c->max_time_steps = 1;
    c->time_mode = CFDG_TIME_STEADY;
    c->bdf_order = 2;
    c->newton_operator = CFDG_NEWTON_PICARD;
    c->jf_max_iterations = 60;
    c->jf_rel_tol = 1.0e-2;
    c->jf_eps = 1.0e-7;
    c->jf_max_change = 0.2;
    c->cfl_ser_max = 0.0;
    c->jf_krylov = CFDG_JF_GMRES;
    c->jf_restart = 30;
    c->jf_accept = 0.5;
}

// ------------------------------------------------------------------ meshes
int cfdg_mesh_generate(const cfdg_mesh_spec* spec, cfdg_host_mesh** out) {
    if (!spec || !out) return CFDG_ERR_INVALID;
    *out = nullptr;
    return guarded([&] {
        auto* m = new cfdg_host_mesh();
        std::string err;
        const int st = cfdg::generate_mesh(*spec, m->mesh, err);
        if (st != CFDG_OK) {
            delete m;
            throw cfdg::Failure{st, err};
        }
        *out = m;
    });
}

int cfdg_host_mesh_view(const cfdg_host_mesh* mesh, cfdg_mesh_host* view) {
    if (!mesh || !view) return CFDG_ERR_INVALID;
    mesh->mesh.view(*view);
    return CFDG_OK;
}

int cfdg_host_mesh_free(cfdg_host_mesh* mesh) {
    delete mesh;
    return CFDG_OK;
}

int cfdg_mesh_compute_geometry(cfdg_host_mesh* mesh) {
    if (!mesh) return CFDG_ERR_INVALID;
    return guarded([&] {
        std::string err;
        if (!cfdg::compute_geometry(mesh->mesh, err)) throw cfdg::Failure{CFDG_ERR_MESH, err};
    });
}

// ------------------------------------------------------------------ solver
int cfdg_solver_create(int device, const cfdg_mesh_host* mesh, const cfdg_config* cfg, const cfdg_bc_desc* bcs,
                       int32_t n_bcs, cfdg_solver** out) {
    if (!mesh || !cfg || !out || (n_bcs > 0 && !bcs) || n_bcs < 0) return CFDG_ERR_INVALID;
    *out = nullptr;
    const int dev = require_device(device);
    if (dev != CFDG_OK) return dev;
    return guarded([&] {
        auto* s = new cfdg_solver{nullptr, device};
        try {
            s->impl = new cfdg::Solver(device, *mesh, *cfg, bcs, n_bcs);
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
    });
}

int cfdg_solver_destroy(cfdg_solver* s) {
    if (!s) return CFDG_OK;
    const int st = guarded([&] { delete s->impl; });
    delete s;
    return st;
}

#define CFDG_SOLVER_CALL(s, ...)                     \
    if (!(s) || !(s)->impl) return CFDG_ERR_INVALID; \
    return guarded([&] { cudaSetDevice((s)->device); __VA_ARGS__; })

int cfdg_solver_init_fields(cfdg_solver* s) { CFDG_SOLVER_CALL(s, s->impl->init_fields()); }

int cfdg_solver_set_state(cfdg_solver* s, const double* u_h, int64_t ld) {
    if (!u_h) return CFDG_ERR_INVALID;
    CFDG_SOLVER_CALL(s, s->impl->set_state_host(u_h, ld));
}

int cfdg_solver_get_field(cfdg_solver* s, int32_t field, double* out_h, int64_t count) {
    if (!out_h) return CFDG_ERR_INVALID;
    CFDG_SOLVER_CALL(s, s->impl->get_field(field, out_h, count));
}

int cfdg_solver_sizes(const cfdg_solver* s, int64_t* sizes_h) {
    if (!s || !s->impl || !sizes_h) return CFDG_ERR_INVALID;
    s->impl->sizes(sizes_h);
    return CFDG_OK;
}

int cfdg_evaluate_residual(cfdg_solver* s) {
    CFDG_SOLVER_CALL(s, s->impl->evaluate_residual(); cfdg::cuda_check(cudaStreamSynchronize(s->impl->stream()), "sync"));
}

int cfdg_solver_stage(cfdg_solver* s, int32_t stage) {
    CFDG_SOLVER_CALL(s, s->impl->stage(stage); cfdg::cuda_check(cudaStreamSynchronize(s->impl->stream()), "sync"));
}

int cfdg_compute_dt(cfdg_solver* s, double cfl) {
    CFDG_SOLVER_CALL(s, s->impl->compute_dt(cfl); cfdg::cuda_check(cudaStreamSynchronize(s->impl->stream()), "sync"));
}

int cfdg_assemble_jacobian(cfdg_solver* s) {
    CFDG_SOLVER_CALL(s, s->impl->assemble_jacobian(); cfdg::cuda_check(cudaStreamSynchronize(s->impl->stream()), "sync"));
}

int cfdg_linear_solve(cfdg_solver* s, cfdg_krylov_result* out_h) {
    CFDG_SOLVER_CALL(s, {
        const cfdg_krylov_result r = s->impl->linear_solve();
        if (out_h) *out_h = r;
    });
}

int cfdg_newton_step(cfdg_solver* s, double cfl, cfdg_step_result* out_h) {
    CFDG_SOLVER_CALL(s, {
        const cfdg_step_result r = s->impl->newton_step(cfl);
        if (out_h) *out_h = r;
    });
}

int cfdg_solver_freeze_limiter(cfdg_solver* s, int32_t frozen) {
    CFDG_SOLVER_CALL(s, { s->impl->freeze_limiter(frozen != 0); });
}

int cfdg_solver_set_limiter(cfdg_solver* s, const double* phi_h, int64_t count) {
    if (!phi_h) return CFDG_ERR_INVALID;
    CFDG_SOLVER_CALL(s, s->impl->set_limiter(phi_h, count));
}

int cfdg_residual_norms(cfdg_solver* s, double* l2_h) {
    if (!l2_h) return CFDG_ERR_INVALID;
    CFDG_SOLVER_CALL(s, s->impl->residual_norms(l2_h));
}

int cfdg_run_steady(cfdg_solver* s, cfdg_run_result* out_h) {
    CFDG_SOLVER_CALL(s, {
        const cfdg_run_result r = s->impl->run_steady();
        if (out_h) *out_h = r;
    });
}

int cfdg_run_unsteady(cfdg_solver* s, cfdg_unsteady_result* out_h) {
    CFDG_SOLVER_CALL(s, {
        const cfdg_unsteady_result r = s->impl->run_unsteady();
        if (out_h) *out_h = r;
    });
}

int cfdg_solver_write_vtu(cfdg_solver* s, const cfdg_mesh_host* mesh_h, const char* outdir, const char* stem) {
    if (!mesh_h || !outdir || !stem) return CFDG_ERR_INVALID;
    CFDG_SOLVER_CALL(s, s->impl->write_vtu(*mesh_h, outdir, stem));
}

int cfdg_solver_reset_time_levels(cfdg_solver* s) { CFDG_SOLVER_CALL(s, s->impl->reset_time_levels()); }

void* cfdg_solver_stream(cfdg_solver* s) { return (s && s->impl) ? static_cast<void*>(s->impl->stream()) : nullptr; }

int64_t cfdg_solver_launch_count(const cfdg_solver* s) { return (s && s->impl) ? s->impl->launches() : -1; }

int cfdg_solver_profile(cfdg_solver* s, int32_t enable) {
    CFDG_SOLVER_CALL(s, {
        cfdg::cuda_check(cudaStreamSynchronize(s->impl->stream()), "sync");
        s->impl->profiler().collect();
        s->impl->profiler().enable(enable != 0);
    });
}

int cfdg_solver_profile_read(cfdg_solver* s, double* ms_h, int64_t* launches_h, double* bytes_h) {
    if (!ms_h || !launches_h) return CFDG_ERR_INVALID;
    CFDG_SOLVER_CALL(s, {
        cfdg::cuda_check(cudaStreamSynchronize(s->impl->stream()), "sync");
        s->impl->profiler().collect();
        for (int c = 0; c < CFDG_KCAT_COUNT; ++c) {
            ms_h[c] = s->impl->profiler().ms[c];
            launches_h[c] = s->impl->profiler().count[c];
            if (bytes_h) bytes_h[c] = s->impl->profiler().bytes[c];
        }
    });
}

int cfdg_solver_sgs_info(const cfdg_solver* s, int32_t* fwd, int32_t* bwd) {
    if (!s || !s->impl || !fwd || !bwd) return CFDG_ERR_INVALID;
    *fwd = s->impl->system().groups_fwd();
    *bwd = s->impl->system().groups_bwd();
    return CFDG_OK;
}

// -------------------------------------------------------------- linalg
int cfdg_bsr_create(int device, int32_t n_rows, int32_t bs, const int32_t* row_ptr_h, const int32_t* cols_h,
                    int32_t precision, cfdg_bsr** out) {
    if (!out || !row_ptr_h || (!cols_h && n_rows > 0)) return CFDG_ERR_INVALID;
    *out = nullptr;
    const int dev = require_device(device);
    if (dev != CFDG_OK) return dev;
    return guarded([&] {
        cfdg::cuda_check(cudaSetDevice(device), "cudaSetDevice");
        auto* a = new cfdg_bsr{nullptr, nullptr, device};
        try {
            cfdg::cuda_check(cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            a->impl = new cfdg::BsrSystem(device, n_rows, bs, row_ptr_h, cols_h, precision, a->stream);
            cfdg::cuda_check(cudaStreamSynchronize(a->stream), "sync");
        } catch (...) {
            if (a->stream) cudaStreamDestroy(a->stream);
            delete a;
            throw;
        }
        *out = a;
    });
}

int cfdg_bsr_destroy(cfdg_bsr* a) {
    if (!a) return CFDG_OK;
    const int st = guarded([&] {
        delete a->impl;
        if (a->stream) cudaStreamDestroy(a->stream);
    });
    delete a;
    return st;
}

#define CFDG_BSR_CALL(a, ...)                        \
    if (!(a) || !(a)->impl) return CFDG_ERR_INVALID; \
    return guarded([&] { cudaSetDevice((a)->device); __VA_ARGS__; })

int cfdg_bsr_set_values(cfdg_bsr* a, const double* values_h) {
    if (!values_h) return CFDG_ERR_INVALID;
    CFDG_BSR_CALL(a, a->impl->set_values_host(values_h); cfdg::cuda_check(cudaStreamSynchronize(a->stream), "sync"));
}

int cfdg_bsr_spmv(cfdg_bsr* a, const double* x_d, double* y_d, double alpha, double beta) {
    if (!x_d || !y_d) return CFDG_ERR_INVALID;
    CFDG_BSR_CALL(a, a->impl->spmv(x_d, y_d, alpha, beta); cfdg::cuda_check(cudaStreamSynchronize(a->stream), "sync"));
}

namespace {
struct HostVec {
    double* d = nullptr;
    ~HostVec() {
        if (d) cudaFree(d);
    }
    void make(std::size_t n, cudaStream_t s, const double* src) {
        cfdg::cuda_check(cudaMalloc(reinterpret_cast<void**>(&d), sizeof(double) * (n ? n : 1)), "cudaMalloc");
        if (src && n) cfdg::cuda_check(cudaMemcpyAsync(d, src, sizeof(double) * n, cudaMemcpyHostToDevice, s), "H2D");
        else cfdg::cuda_check(cudaMemsetAsync(d, 0, sizeof(double) * (n ? n : 1), s), "memset");
    }
    void get(double* dst, std::size_t n, cudaStream_t s) {
        if (n) cfdg::cuda_check(cudaMemcpyAsync(dst, d, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "D2H");
        cfdg::cuda_check(cudaStreamSynchronize(s), "sync");
    }
};
}  // namespace

int cfdg_bsr_spmv_host(cfdg_bsr* a, const double* x_h, double* y_h, double alpha, double beta) {
    if (!x_h || !y_h) return CFDG_ERR_INVALID;
    CFDG_BSR_CALL(a, {
        const std::size_t N = static_cast<std::size_t>(a->impl->n()) * a->impl->bs();
        HostVec x, y;
        x.make(N, a->stream, x_h);
        y.make(N, a->stream, y_h);
        a->impl->spmv(x.d, y.d, alpha, beta);
        y.get(y_h, N, a->stream);
    });
}

int cfdg_sgs_setup(cfdg_bsr* a, int32_t ordering, int32_t sweeps) {
    CFDG_BSR_CALL(a, a->impl->sgs_setup(ordering, sweeps));
}

int cfdg_sgs_apply(cfdg_bsr* a, const double* r_d, double* z_d) {
    if (!r_d || !z_d) return CFDG_ERR_INVALID;
    CFDG_BSR_CALL(a, a->impl->sgs_apply(r_d, z_d, nullptr); cfdg::cuda_check(cudaStreamSynchronize(a->stream), "sync"));
}

int cfdg_sgs_apply_host(cfdg_bsr* a, const double* r_h, double* z_h) {
    if (!r_h || !z_h) return CFDG_ERR_INVALID;
    CFDG_BSR_CALL(a, {
        const std::size_t N = static_cast<std::size_t>(a->impl->n()) * a->impl->bs();
        HostVec r, z;
        r.make(N, a->stream, r_h);
        z.make(N, a->stream, nullptr);
        a->impl->sgs_apply(r.d, z.d, nullptr);
        z.get(z_h, N, a->stream);
    });
}

int cfdg_bicgstab(cfdg_bsr* a, int32_t precond, double rel_tol, double abs_tol, int32_t max_it, double* x_d,
                  const double* b_d, cfdg_krylov_result* out_h) {
    if (!x_d || !b_d) return CFDG_ERR_INVALID;
    CFDG_BSR_CALL(a, {
        const cfdg_krylov_result r = a->impl->bicgstab(precond, rel_tol, abs_tol, max_it, x_d, b_d);
        if (out_h) *out_h = r;
    });
}

int cfdg_bicgstab_host(cfdg_bsr* a, int32_t precond, double rel_tol, double abs_tol, int32_t max_it, double* x_h,
                       const double* b_h, cfdg_krylov_result* out_h) {
    if (!x_h || !b_h) return CFDG_ERR_INVALID;
    CFDG_BSR_CALL(a, {
        const std::size_t N = static_cast<std::size_t>(a->impl->n()) * a->impl->bs();
        HostVec x, b;
        x.make(N, a->stream, x_h);
        b.make(N, a->stream, b_h);
        const cfdg_krylov_result r = a->impl->bicgstab(precond, rel_tol, abs_tol, max_it, x.d, b.d);
        x.get(x_h, N, a->stream);
        if (out_h) *out_h = r;
    });
}

int cfdg_gmres(cfdg_bsr* a, int32_t precond, double rel_tol, double abs_tol, int32_t max_it, int32_t restart,
               double* x_d, const double* b_d, cfdg_krylov_result* out_h) {
    if (!x_d || !b_d) return CFDG_ERR_INVALID;
    CFDG_BSR_CALL(a, {
        const cfdg_krylov_result r = a->impl->gmres(precond, rel_tol, abs_tol, max_it, restart, x_d, b_d);
        if (out_h) *out_h = r;
    });
}

int cfdg_gmres_host(cfdg_bsr* a, int32_t precond, double rel_tol, double abs_tol, int32_t max_it, int32_t restart,
                    double* x_h, const double* b_h, cfdg_krylov_result* out_h) {
    if (!x_h || !b_h) return CFDG_ERR_INVALID;
    CFDG_BSR_CALL(a, {
        const std::size_t N = static_cast<std::size_t>(a->impl->n()) * a->impl->bs();
        HostVec x, b;
        x.make(N, a->stream, x_h);
        b.make(N, a->stream, b_h);
        const cfdg_krylov_result r = a->impl->gmres(precond, rel_tol, abs_tol, max_it, restart, x.d, b.d);
        x.get(x_h, N, a->stream);
        if (out_h) *out_h = r;
    });
}

/* ----------------------------------------------------- learned guess */
int cfdg_tc_selftest(int device, int32_t n, int32_t k, const uint16_t* a_h, const uint16_t* b_h, float* d_h) {
    if (!a_h || !b_h || !d_h) return CFDG_ERR_INVALID;
    if (!(n == 16 || n == 32 || n == 48 || n == 64) || k < 16 || k > 128 || k % 16) return CFDG_ERR_INVALID;
    const int dev = require_device(device);
    if (dev != CFDG_OK) return dev;
    return guarded([&] {
        cfdg::cuda_check(cudaSetDevice(device), "cudaSetDevice");
        uint16_t *A = nullptr, *B = nullptr;
        float* D = nullptr;
        int* err = nullptr;
        auto release = [&] {
            cudaFree(A);
            cudaFree(B);
            cudaFree(D);
            cudaFree(err);
        };
        try {
            cfdg::cuda_check(cudaMalloc(reinterpret_cast<void**>(&A), 128 * k * 2), "cudaMalloc");
            cfdg::cuda_check(cudaMalloc(reinterpret_cast<void**>(&B), 64 * k * 2), "cudaMalloc");
            cfdg::cuda_check(cudaMalloc(reinterpret_cast<void**>(&D), 128 * 64 * 4), "cudaMalloc");
            cfdg::cuda_check(cudaMalloc(reinterpret_cast<void**>(&err), 4), "cudaMalloc");
            cfdg::cuda_check(cudaMemset(err, 0, 4), "memset");
            cfdg::cuda_check(cudaMemcpy(A, a_h, 128 * k * 2, cudaMemcpyHostToDevice), "H2D");
            cfdg::cuda_check(cudaMemcpy(B, b_h, n * k * 2, cudaMemcpyHostToDevice), "H2D");
            cfdg::launch_tc_selftest(A, B, D, n, k, err, nullptr);
            cfdg::cuda_check(cudaGetLastError(), "selftest launch");
            cfdg::cuda_check(cudaDeviceSynchronize(), "selftest");
            int e = 0;
            cfdg::cuda_check(cudaMemcpy(&e, err, 4, cudaMemcpyDeviceToHost), "D2H");
            if (e) throw cfdg::Failure{CFDG_ERR_CUDA, "tensor-core self-test: MMA completion wait timed out"};
            cfdg::cuda_check(cudaMemcpy(d_h, D, 128 * n * 4, cudaMemcpyDeviceToHost), "D2H");
        } catch (...) {
            release();
            throw;
        }
        release();
    });
}

int cfdg_mlp_create(int device, int32_t nvars, uint64_t seed, cfdg_mlp** out) {
    if (!out) return CFDG_ERR_INVALID;
    *out = nullptr;
    const int dev = require_device(device);
    if (dev != CFDG_OK) return dev;
    return guarded([&] {
        cfdg::cuda_check(cudaSetDevice(device), "cudaSetDevice");
        auto* m = new cfdg_mlp{nullptr, nullptr, device};
        try {
            cfdg::cuda_check(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "cudaStreamCreate");
            m->impl = new cfdg::Mlp(device, nvars, seed);
        } catch (...) {
            if (m->stream) cudaStreamDestroy(m->stream);
            delete m;
            throw;
        }
        *out = m;
    });
}

int cfdg_mlp_destroy(cfdg_mlp* m) {
    if (!m) return CFDG_OK;
    const int st = guarded([&] {
        cudaSetDevice(m->device);
        delete m->impl;
        if (m->stream) cudaStreamDestroy(m->stream);
    });
    delete m;
    return st;
}

#define CFDG_MLP_CALL(m, ...)                        \
    if (!(m) || !(m)->impl) return CFDG_ERR_INVALID; \
    return guarded([&] { cudaSetDevice((m)->device); __VA_ARGS__; })

int32_t cfdg_mlp_param_count(void) { return cfdg::kMlpParams; }

int cfdg_mlp_get_params(cfdg_mlp* m, float* out_h, int64_t count) {
    if (!out_h || count < cfdg::kMlpParams) return CFDG_ERR_INVALID;
    CFDG_MLP_CALL(m, m->impl->get_params(out_h));
}

int cfdg_mlp_set_params(cfdg_mlp* m, const float* p_h, int64_t count) {
    if (!p_h || count < cfdg::kMlpParams) return CFDG_ERR_INVALID;
    CFDG_MLP_CALL(m, m->impl->set_params(p_h));
}

int cfdg_mlp_forward(cfdg_mlp* m, const uint16_t* feat_d, int64_t rows, const double* scale_d, double* out_d) {
    if (!feat_d || !scale_d || !out_d || rows < 0) return CFDG_ERR_INVALID;
    CFDG_MLP_CALL(m, {
        m->impl->forward(feat_d, rows, scale_d, out_d, m->stream);
        cfdg::cuda_check(cudaStreamSynchronize(m->stream), "sync");
    });
}

int cfdg_mlp_forward_host(cfdg_mlp* m, const uint16_t* feat_h, int64_t rows, double* out_h) {
    if (!feat_h || !out_h || rows < 0) return CFDG_ERR_INVALID;
    CFDG_MLP_CALL(m, {
        const int nv = m->impl->nvars();
        uint16_t* F = nullptr;
        double *O = nullptr, *S = nullptr;
        auto release = [&] {
            cudaFree(F);
            cudaFree(O);
            cudaFree(S);
        };
        try {
            cfdg::cuda_check(cudaMalloc(reinterpret_cast<void**>(&F), std::max<int64_t>(rows, 1) * cfdg::kMlpIn * 2),
                             "cudaMalloc");
            cfdg::cuda_check(cudaMalloc(reinterpret_cast<void**>(&O), std::max<int64_t>(rows, 1) * nv * 8), "cudaMalloc");
            cfdg::cuda_check(cudaMalloc(reinterpret_cast<void**>(&S), 8 * 8), "cudaMalloc");
            const double ones[8] = {1, 1, 1, 1, 1, 1, 1, 1};
            cfdg::cuda_check(cudaMemcpy(S, ones, sizeof(ones), cudaMemcpyHostToDevice), "H2D");
            cfdg::cuda_check(cudaMemcpy(F, feat_h, rows * cfdg::kMlpIn * 2, cudaMemcpyHostToDevice), "H2D");
            m->impl->forward(F, rows, S, O, m->stream);
            cfdg::cuda_check(cudaStreamSynchronize(m->stream), "sync");
            cfdg::cuda_check(cudaMemcpy(out_h, O, rows * nv * 8, cudaMemcpyDeviceToHost), "D2H");
        } catch (...) {
            release();
            throw;
        }
        release();
    });
}

int cfdg_mlp_gradient_host(cfdg_mlp* m, const uint16_t* x_h, const float* t_h, int64_t rows, float* loss_h,
                           float* grad_h) {
    if (!x_h || !t_h || rows <= 0) return CFDG_ERR_INVALID;
    CFDG_MLP_CALL(m, {
        cfdg::Dataset tmp(m->device, m->impl->nvars(), rows);
        tmp.append_host(x_h, t_h, rows);
        const float l = m->impl->gradient(tmp.X(), tmp.T(), rows, grad_h, m->stream);
        if (loss_h) *loss_h = l;
    });
}

int cfdg_mlp_train(cfdg_mlp* m, cfdg_dataset* ds, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                   float* loss_h) {
    if (!ds || !ds->impl || epochs < 1 || !(lr > 0.0f)) return CFDG_ERR_INVALID;
    CFDG_MLP_CALL(m, {
        const float l = m->impl->train(*ds->impl, epochs, batch, lr, seed, m->stream);
        if (loss_h) *loss_h = l;
    });
}

int cfdg_dataset_create(int device, int32_t nvars, int64_t capacity, cfdg_dataset** out) {
    if (!out) return CFDG_ERR_INVALID;
    *out = nullptr;
    const int dev = require_device(device);
    if (dev != CFDG_OK) return dev;
    return guarded([&] {
        auto* d = new cfdg_dataset{nullptr, device};
        try {
            d->impl = new cfdg::Dataset(device, nvars, capacity);
        } catch (...) {
            delete d;
            throw;
        }
        *out = d;
    });
}

int cfdg_dataset_destroy(cfdg_dataset* d) {
    if (!d) return CFDG_OK;
    const int st = guarded([&] {
        cudaSetDevice(d->device);
        delete d->impl;
    });
    delete d;
    return st;
}

int cfdg_dataset_size(const cfdg_dataset* d, int64_t* size_h) {
    if (!d || !d->impl || !size_h) return CFDG_ERR_INVALID;
    *size_h = d->impl->size();
    return CFDG_OK;
}

int cfdg_dataset_clear(cfdg_dataset* d) {
    if (!d || !d->impl) return CFDG_ERR_INVALID;
    d->impl->clear();
    return CFDG_OK;
}

int cfdg_dataset_append_host(cfdg_dataset* d, const uint16_t* x_h, const float* t_h, int64_t rows) {
    if (!d || !d->impl || !x_h || !t_h || rows < 0) return CFDG_ERR_INVALID;
    return guarded([&] {
        cudaSetDevice(d->device);
        d->impl->append_host(x_h, t_h, rows);
    });
}

int cfdg_dataset_read_host(const cfdg_dataset* d, uint16_t* x_h, float* t_h, int64_t rows) {
    if (!d || !d->impl || rows < 0) return CFDG_ERR_INVALID;
    return guarded([&] {
        cudaSetDevice(d->device);
        d->impl->read_host(x_h, t_h, rows);
    });
}

int cfdg_solver_attach_guess(cfdg_solver* s, cfdg_mlp* m) {
    if (m && !m->impl) return CFDG_ERR_INVALID;
    CFDG_SOLVER_CALL(s, s->impl->attach_guess(m ? m->impl : nullptr));
}

int cfdg_solver_attach_dataset(cfdg_solver* s, cfdg_dataset* d, int32_t stride) {
    if (d && !d->impl) return CFDG_ERR_INVALID;
    CFDG_SOLVER_CALL(s, s->impl->attach_dataset(d ? d->impl : nullptr, stride));
}

// ------------------------------------------------- gradient / limiter operators
int cfdg_recon_create(int device, const cfdg_mesh_host* mesh_h, int32_t gradient, int32_t limiter, double venkat_k,
                      cfdg_recon** out) {
    if (!mesh_h || !out) return CFDG_ERR_INVALID;
    *out = nullptr;
    const int dv = require_device(device);
    if (dv != CFDG_OK) return dv;
    return guarded([&] {
        auto* r = new cfdg_recon{nullptr};
        try {
            r->impl = new cfdg::ReconOperator(device, *mesh_h, gradient, limiter, venkat_k);
        } catch (...) {
            delete r;
            throw;
        }
        *out = r;
    });
}

int cfdg_recon_destroy(cfdg_recon* r) {
    if (!r) return CFDG_OK;
    if (r->impl) cudaSetDevice(r->impl->device());
    delete r->impl;
    delete r;
    return CFDG_OK;
}

int cfdg_gradient(cfdg_recon* r, const double* const* q_d, double* const* gx_d, double* const* gy_d,
                  double* const* gz_d, int32_t nvars, void* stream) {
    if (!r || !r->impl) return CFDG_ERR_INVALID;
    return guarded([&] { r->impl->gradient(q_d, gx_d, gy_d, gz_d, nvars, static_cast<cudaStream_t>(stream)); });
}

int cfdg_limiter(cfdg_recon* r, const double* const* q_d, const double* const* gx_d, const double* const* gy_d,
                 const double* const* gz_d, double* const* phi_d, int32_t nvars, void* stream) {
    if (!r || !r->impl) return CFDG_ERR_INVALID;
    return guarded([&] { r->impl->limiter(q_d, gx_d, gy_d, gz_d, phi_d, nvars, static_cast<cudaStream_t>(stream)); });
}

// ------------------------------------------------------ partitions and halos
int cfdg_halo_create(const cfdg_mesh_host* mesh_h, int32_t nparts, const int32_t* part_h, int32_t rank,
                     cfdg_halo** out) {
    if (!mesh_h || !out) return CFDG_ERR_INVALID;
    *out = nullptr;
    return guarded([&] {
        cfdg::HostMesh hm;
        hm.from_view(*mesh_h);
        auto* h = new cfdg_halo{};
        try {
            cfdg::build_halo_plan(hm, nparts, part_h, rank, h->plan);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int cfdg_halo_destroy(cfdg_halo* h) {
    if (!h) return CFDG_OK;
    if (h->plan.device >= 0) cudaSetDevice(h->plan.device);
    delete h;
    return CFDG_OK;
}

int cfdg_halo_sizes(const cfdg_halo* h, int64_t* sizes_h) {
    if (!h || !sizes_h) return CFDG_ERR_INVALID;
    const cfdg::HaloPlan& p = h->plan;
    sizes_h[0] = p.n_own;
    sizes_h[1] = p.n_local;
    sizes_h[2] = static_cast<int64_t>(p.nb_ranks.size());
    sizes_h[3] = static_cast<int64_t>(p.send_owned_local.size());
    sizes_h[4] = static_cast<int64_t>(p.recv_ghost_local.size());
    return CFDG_OK;
}

int cfdg_halo_get(const cfdg_halo* h, int32_t what, int32_t* out_h, int64_t count) {
    if (!h || !out_h) return CFDG_ERR_INVALID;
    const cfdg::HaloPlan& p = h->plan;
    const std::vector<int32_t>* v = nullptr;
    switch (what) {
        case CFDG_HALO_LOCAL_TO_GLOBAL: v = &p.local_to_global; break;
        case CFDG_HALO_NB_RANKS: v = &p.nb_ranks; break;
        case CFDG_HALO_SEND_OFFSETS: v = &p.send_offsets; break;
        case CFDG_HALO_SEND_OWNED_LOCAL: v = &p.send_owned_local; break;
        case CFDG_HALO_RECV_OFFSETS: v = &p.recv_offsets; break;
        case CFDG_HALO_RECV_GHOST_LOCAL: v = &p.recv_ghost_local; break;
        default: cfdg::set_error("unknown halo array"); return CFDG_ERR_INVALID;
    }
    if (count < static_cast<int64_t>(v->size())) {
        cfdg::set_error("output buffer too small");
        return CFDG_ERR_INVALID;
    }
    std::copy(v->begin(), v->end(), out_h);
    return CFDG_OK;
}


int cfdg_halo_pack(cfdg_halo* h, int device, const double* const* fields_d, int32_t nvars, double* send_d,
                   void* stream) {
    if (!h || !fields_d || (!send_d && !h->plan.send_owned_local.empty())) return CFDG_ERR_INVALID;
    const int st = halo_device_ready(h, device, nvars);
    if (st != CFDG_OK) return st;
    return guarded([&] {
        cfdg::HaloFields f{};
        for (int v = 0; v < nvars; ++v) f.p[v] = const_cast<double*>(fields_d[v]);
        cfdg::launch_halo_pack(static_cast<int32_t>(h->plan.send_owned_local.size()), h->plan.send_d.p, f, nvars,
                               send_d, static_cast<cudaStream_t>(stream));
        cfdg::cuda_check(cudaGetLastError(), "halo pack launch");
    });
}

int cfdg_halo_unpack(cfdg_halo* h, int device, const double* recv_d, int32_t nvars, double* const* fields_d,
                     void* stream) {
    if (!h || !fields_d || (!recv_d && !h->plan.recv_ghost_local.empty())) return CFDG_ERR_INVALID;
    const int st = halo_device_ready(h, device, nvars);
    if (st != CFDG_OK) return st;
    return guarded([&] {
        cfdg::HaloFields f{};
        for (int v = 0; v < nvars; ++v) f.p[v] = fields_d[v];
        cfdg::launch_halo_unpack(static_cast<int32_t>(h->plan.recv_ghost_local.size()), h->plan.recv_d.p, recv_d,
                                 nvars, f, static_cast<cudaStream_t>(stream));
        cfdg::cuda_check(cudaGetLastError(), "halo unpack launch");
    });
}

int cfdg_halo_pack_blocks(cfdg_halo* h, int device, const double* x_d, int32_t bs, double* send_d, void* stream) {
    if (!h || !x_d || (!send_d && !h->plan.send_owned_local.empty())) return CFDG_ERR_INVALID;
    const int st = halo_device_ready(h, device, bs);
    if (st != CFDG_OK) return st;
    return guarded([&] {
        cfdg::launch_halo_pack_blocks(static_cast<int32_t>(h->plan.send_owned_local.size()), h->plan.send_d.p, x_d,
                                      bs, send_d, static_cast<cudaStream_t>(stream));
        cfdg::cuda_check(cudaGetLastError(), "halo pack launch");
    });
}

int cfdg_halo_unpack_blocks(cfdg_halo* h, int device, const double* recv_d, int32_t bs, double* x_d, void* stream) {
    if (!h || !x_d || (!recv_d && !h->plan.recv_ghost_local.empty())) return CFDG_ERR_INVALID;
    const int st = halo_device_ready(h, device, bs);
    if (st != CFDG_OK) return st;
    return guarded([&] {
        cfdg::launch_halo_unpack_blocks(static_cast<int32_t>(h->plan.recv_ghost_local.size()), h->plan.recv_d.p,
                                        recv_d, bs, x_d, static_cast<cudaStream_t>(stream));
        cfdg::cuda_check(cudaGetLastError(), "halo unpack launch");
    });
}

}  // extern "C"
