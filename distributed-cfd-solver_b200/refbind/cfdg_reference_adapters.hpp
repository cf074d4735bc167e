// GPU drop-ins behind the reference solver's own interfaces.
//
// A maintainer of the reference code base includes this header (it is
// compiled against the reference's headers, include/cfd/..., and links
// libcfdg.so) to swap the CPU hot path for the B200 one at the seams the
// reference already has:
//
//   GpuBsrOperator  : linalg::LinearOperator     (include/cfd/linalg/operator.hpp:20-42)
//   GpuSgs          : linalg::Preconditioner     (include/cfd/linalg/preconditioner.hpp:22-28)
//   GpuBiCGSTAB     : linalg::IterativeSolver    (include/cfd/linalg/solver.hpp:23-47)
//   GpuGradient     : gradient::GradientOperator (include/cfd/numerics/gradient/gradient_operator.hpp:16-44)
//   GpuBackwardEuler<Op> : a time policy satisfying TimeIntegrationPolicy
//                     (include/cfd/solver/compressible/time/concepts.hpp:16-28); its advance()
//                     is one whole implicit iteration on the GPU (cfdg_newton_step).
//
// The reference's vectors and fields live in host memory, so each call
// copies its operands to the device and its result back (the linear-algebra
// adapters through the cfdg_*_host entry points, the gradient through
// device staging buffers); the device keeps the matrix, the preconditioner
// factors and the solver state between calls.  Failures follow the
// reference's convention: linalg::fatal / mpi::fatal (MPI_Abort) with the
// library's message.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <span>
#include <string>
#include <vector>

#include "cfd/bc/config.hpp"
#include "cfd/linalg/bsr_matrix.hpp"
#include "cfd/linalg/operator.hpp"
#include "cfd/linalg/preconditioner.hpp"
#include "cfd/linalg/preconditioners.hpp"
#include "cfd/linalg/solver.hpp"
#include "cfd/mesh/aux_connectivity.hpp"
#include "cfd/mesh/aux_geometry.hpp"
#include "cfd/mesh/localmesh.hpp"
#include "cfd/numerics/gradient/gradient_operator.hpp"
#include "cfd/solver/compressible/config.hpp"
#include "cfdg.h"

namespace cfdg::refbind {

namespace linalg = cfd::linalg;
namespace mesh = cfd::mesh;

inline void require(int status, MPI_Comm comm, const char* what) {
    if (status != CFDG_OK) linalg::fatal(comm, std::string(what) + ": " + cfdg_last_error());
}

// cfdg_mesh_host view of a single-partition MeshPart (n_own == n_cells).
// The view points into `mp` and is valid while `mp` is unchanged.
struct MeshView {
    cfdg_mesh_host v{};
    std::vector<uint8_t> cell_type;
    explicit MeshView(const mesh::MeshPart& mp) {
        linalg::check(mp.n_own == mp.n_cells, MPI_COMM_WORLD,
                      "cfdg adapters: one partition per GPU (no ghost cells) is supported");
        cell_type.resize(mp.cell_type.size());
        for (std::size_t c = 0; c < cell_type.size(); ++c) cell_type[c] = static_cast<uint8_t>(mp.cell_type[c]);
        v.n_cells = mp.n_cells;
        v.n_faces = mp.n_faces;
        v.n_inner_faces = mp.n_inner_faces;
        v.n_nodes = mp.n_nodes;
        v.n_patches = static_cast<int32_t>(mp.patches.size());
        v.cell_type = cell_type.data();
        v.cell_nodes_offsets = mp.cell_nodes_offsets.data();
        v.cell_nodes = mp.cell_nodes.data();
        v.node_x = mp.node_x.data();
        v.node_y = mp.node_y.data();
        v.node_z = mp.node_z.data();
        v.cell_centroid_x = mp.cell_centroid_x.data();
        v.cell_centroid_y = mp.cell_centroid_y.data();
        v.cell_centroid_z = mp.cell_centroid_z.data();
        v.cell_volume = mp.cell_volume.data();
        v.face_owner = mp.face_owner.data();
        v.face_neigh = mp.face_neigh.data();
        v.face_patch = mp.face_patch.data();
        v.face_nodes_offsets = mp.face_nodes_offsets.data();
        v.face_nodes = mp.face_nodes.data();
        v.face_centroid_x = mp.face_centroid_x.data();
        v.face_centroid_y = mp.face_centroid_y.data();
        v.face_centroid_z = mp.face_centroid_z.data();
        v.face_normal_x = mp.face_normal_x.data();
        v.face_normal_y = mp.face_normal_y.data();
        v.face_normal_z = mp.face_normal_z.data();
        v.face_area = mp.face_area.data();
    }
};

// --------------------------------------------------------------- linalg
// The reference BsrMatrix's structure and values on the device.  upload()
// copies the values after each assembly; apply() is y = alpha A x + beta y.
class GpuBsrOperator final : public linalg::LinearOperator {
public:
    GpuBsrOperator(const linalg::BsrMatrix& A, int device = 0, int precision = CFDG_PREC_FP64) : A_(A) {
        const MPI_Comm comm = A.layout().comm();
        linalg::check(A.layout().ghostSize() == 0, comm, "GpuBsrOperator: one partition per GPU (no ghost columns)");
        require(cfdg_bsr_create(device, A.localRows(), A.blockSize(), A.rowPtr().data(), A.cols().data(), precision,
                                &h_),
                comm, "GpuBsrOperator");
        upload();
    }
    ~GpuBsrOperator() override { cfdg_bsr_destroy(h_); }
    GpuBsrOperator(const GpuBsrOperator&) = delete;
    GpuBsrOperator& operator=(const GpuBsrOperator&) = delete;

    void upload() { require(cfdg_bsr_set_values(h_, A_.valuesData()), A_.layout().comm(), "GpuBsrOperator::upload"); }

    cfd::GlobalIndex globalRows() const override { return A_.globalRows(); }
    cfd::LocalIndex localRows() const override { return A_.localRows(); }
    int blockSize() const override { return A_.blockSize(); }
    const linalg::VectorLayout& layout() const override { return A_.layout(); }
    linalg::Vector makeVector() const override { return A_.makeVector(); }
    void apply(const linalg::Vector& x, linalg::Vector& y, double alpha = 1.0, double beta = 0.0) const override {
        require(cfdg_bsr_spmv_host(h_, x.data(), y.data(), alpha, beta), A_.layout().comm(), "GpuBsrOperator::apply");
    }

    cfdg_bsr* handle() const { return h_; }
    const linalg::BsrMatrix& matrix() const { return A_; }

private:
    const linalg::BsrMatrix& A_;
    cfdg_bsr* h_ = nullptr;
};

// SGS on the device: setup() is the block LU of the diagonal, apply() one
// symmetric sweep from z = 0.  ordering CFDG_SGS_LEVEL performs the
// reference's sequential sweep exactly (level-scheduled); CFDG_SGS_COLOR a
// multicolour sweep.  setup() takes a GpuBsrOperator, or a BsrMatrix which it
// then uploads itself.
class GpuSgs final : public linalg::Preconditioner {
public:
    explicit GpuSgs(int ordering = CFDG_SGS_LEVEL, int sweeps = 1, int device = 0)
        : ordering_(ordering), sweeps_(sweeps), device_(device) {}

    void setup(const linalg::LinearOperator& op) override {
        if (const auto* g = dynamic_cast<const GpuBsrOperator*>(&op)) {
            op_ = g;
        } else {
            const auto* A = dynamic_cast<const linalg::BsrMatrix*>(&op);
            linalg::check(A != nullptr, op.layout().comm(), "GpuSgs::setup: a BSR operator is required");
            if (!own_ || &own_->matrix() != A) own_ = std::make_unique<GpuBsrOperator>(*A, device_);
            else own_->upload();
            op_ = own_.get();
        }
        require(cfdg_sgs_setup(op_->handle(), ordering_, sweeps_), op.layout().comm(), "GpuSgs::setup");
    }
    void apply(const linalg::Vector& r, linalg::Vector& z) const override {
        require(cfdg_sgs_apply_host(op_->handle(), r.data(), z.data()), r.layout().comm(), "GpuSgs::apply");
    }
    const GpuBsrOperator* op() const { return op_; }

private:
    int ordering_, sweeps_, device_;
    const GpuBsrOperator* op_ = nullptr;
    std::unique_ptr<GpuBsrOperator> own_;
};

// BiCGSTAB on the device (right-preconditioned, the reference's recurrences,
// scalars and inner products on the device): A a GpuBsrOperator, M a GpuSgs
// set up on it or an IdentityPreconditioner; x holds the initial guess.
// The operator and preconditioner checks of the GPU Krylov solvers: a
// GpuBsrOperator, and GpuSgs set up on it or the identity.
inline int gpu_krylov_precond(const linalg::LinearOperator& A, const linalg::Preconditioner& M, const char* who,
                              const GpuBsrOperator*& op) {
    const MPI_Comm comm = A.layout().comm();
    op = dynamic_cast<const GpuBsrOperator*>(&A);
    linalg::check(op != nullptr, comm, std::string(who) + ": the operator must be a GpuBsrOperator");
    if (const auto* sgs = dynamic_cast<const GpuSgs*>(&M)) {
        linalg::check(sgs->op() == op, comm, std::string(who) + ": the GpuSgs was set up on another operator");
        return CFDG_PC_SGS;
    }
    linalg::check(dynamic_cast<const linalg::IdentityPreconditioner*>(&M) != nullptr, comm,
                  std::string(who) + ": GpuSgs or IdentityPreconditioner");
    return CFDG_PC_NONE;
}

inline linalg::IterationResult gpu_krylov_result(const cfdg_krylov_result& r) {
    linalg::IterationResult out;
    out.status = r.status == CFDG_KRYLOV_CONVERGED   ? linalg::SolverStatus::Converged
                 : r.status == CFDG_KRYLOV_DIVERGED ? linalg::SolverStatus::Diverged
                                                     : linalg::SolverStatus::MaxIterations;
    out.iterations = r.iterations;
    out.initial_residual = r.initial_residual;
    out.final_residual = r.final_residual;
    return out;
}

class GpuBiCGSTAB final : public linalg::IterativeSolver {
public:
    const char* name() const override { return "BiCGSTAB (cfdg, GPU)"; }
    linalg::IterationResult solve(const linalg::LinearOperator& A, const linalg::Preconditioner& M,
                                  linalg::Vector& x, const linalg::Vector& b) override {
        const GpuBsrOperator* op = nullptr;
        const int precond = gpu_krylov_precond(A, M, "GpuBiCGSTAB", op);
        cfdg_krylov_result r{};
        require(cfdg_bicgstab_host(op->handle(), precond, params_.relative_tolerance, params_.absolute_tolerance,
                                   params_.max_iterations, x.data(), b.data(), &r),
                A.layout().comm(), "GpuBiCGSTAB::solve");
        last_ = gpu_krylov_result(r);
        return last_;
    }
};

// Restarted GMRES(restart) with right preconditioning behind the same
// IterativeSolver interface (not in the reference: the Krylov method of the
// library's Jacobian-free solves, offered here for any operator).
class GpuGmres final : public linalg::IterativeSolver {
public:
    explicit GpuGmres(int restart = 30) : restart_(restart) {}
    const char* name() const override { return "GMRES (cfdg, GPU)"; }
    linalg::IterationResult solve(const linalg::LinearOperator& A, const linalg::Preconditioner& M,
                                  linalg::Vector& x, const linalg::Vector& b) override {
        const GpuBsrOperator* op = nullptr;
        const int precond = gpu_krylov_precond(A, M, "GpuGmres", op);
        cfdg_krylov_result r{};
        require(cfdg_gmres_host(op->handle(), precond, params_.relative_tolerance, params_.absolute_tolerance,
                                params_.max_iterations, restart_, x.data(), b.data(), &r),
                A.layout().comm(), "GpuGmres::solve");
        last_ = gpu_krylov_result(r);
        return last_;
    }

private:
    int restart_;
};

// ------------------------------------------------------------- gradient
// Least-squares cell gradient (face or vertex-neighbour stencil, the
// reference's LSQ set-up) on the device; the fields are copied through
// device staging buffers sized at setup.
class GpuGradient final : public cfd::numerics::gradient::GradientOperator {
public:
    explicit GpuGradient(int stencil = CFDG_GRAD_LSQ_NODE, int device = 0) : stencil_(stencil), device_(device) {}
    ~GpuGradient() override {
        cfdg_recon_destroy(r_);
        if (buf_) cudaFree(buf_);
    }
    GpuGradient(const GpuGradient&) = delete;
    GpuGradient& operator=(const GpuGradient&) = delete;

    void setup(const mesh::MeshPart& m, mesh::MeshAuxConnectivity& /*aux_conn*/) override {
        const MeshView view(m);
        cfdg_recon_destroy(r_);
        r_ = nullptr;
        require(cfdg_recon_create(device_, &view.v, stencil_, CFDG_LIM_VENKATAKRISHNAN, 0.5, &r_), MPI_COMM_WORLD,
                "GpuGradient::setup");
        n_ = static_cast<std::size_t>(m.n_cells);
    }
    void apply(const double* s, double* gx, double* gy, double* gz, const mesh::MeshPart& m,
               const mesh::MeshAuxConnectivity& aux_conn) const override {
        const double* ss[1] = {s};
        double* xs[1] = {gx};
        double* ys[1] = {gy};
        double* zs[1] = {gz};
        apply_set(ss, xs, ys, zs, m, aux_conn);
    }
    void apply_set(std::span<const double* const> s, std::span<double* const> gx, std::span<double* const> gy,
                   std::span<double* const> gz, const mesh::MeshPart& /*m*/,
                   const mesh::MeshAuxConnectivity& /*aux_conn*/) const override {
        const int nv = static_cast<int>(s.size());
        stage(nv);
        std::vector<const double*> q(nv);
        std::vector<double*> x(nv), y(nv), z(nv);
        for (int v = 0; v < nv; ++v) {
            q[v] = buf_ + (4 * v) * n_;
            x[v] = buf_ + (4 * v + 1) * n_;
            y[v] = buf_ + (4 * v + 2) * n_;
            z[v] = buf_ + (4 * v + 3) * n_;
            copy(const_cast<double*>(q[v]), s[v], cudaMemcpyHostToDevice);
        }
        require(cfdg_gradient(r_, q.data(), x.data(), y.data(), z.data(), nv, nullptr), MPI_COMM_WORLD,
                "GpuGradient::apply_set");
        for (int v = 0; v < nv; ++v) {
            copy(gx[v], x[v], cudaMemcpyDeviceToHost);
            copy(gy[v], y[v], cudaMemcpyDeviceToHost);
            copy(gz[v], z[v], cudaMemcpyDeviceToHost);
        }
    }
    const char* name() const noexcept override { return "LEAST_SQUARES (cfdg, GPU)"; }

private:
    void stage(int nv) const {
        if (nv <= staged_) return;
        if (buf_) cudaFree(buf_);
        buf_ = nullptr;
        if (cudaSetDevice(device_) != cudaSuccess ||
            cudaMalloc(reinterpret_cast<void**>(&buf_), sizeof(double) * 4 * n_ * nv) != cudaSuccess)
            linalg::fatal(MPI_COMM_WORLD, "GpuGradient: device staging allocation failed");
        staged_ = nv;
    }
    void copy(double* dst, const double* src, cudaMemcpyKind k) const {
        if (cudaMemcpy(dst, src, sizeof(double) * n_, k) != cudaSuccess)
            linalg::fatal(MPI_COMM_WORLD, "GpuGradient: copy failed");
    }
    int stencil_, device_;
    cfdg_recon* r_ = nullptr;
    std::size_t n_ = 0;
    mutable double* buf_ = nullptr;
    mutable int staged_ = 0;
};

// ----------------------------------------------------------- time policy
// Options of the GPU iteration and the boundary configuration, which the
// time-policy interface does not pass (set before the Solver is built).
struct GpuTimeOptions {
    int device = 0;
    int precision = CFDG_PREC_FP64;
    int sgs_ordering = CFDG_SGS_LEVEL;   // the reference's sequential sweep
    int jacobian = CFDG_JAC_REFERENCE;
    const cfd::bc::BoundaryConfig* boundaries = nullptr;
};
inline GpuTimeOptions& gpu_time_options() {
    static GpuTimeOptions o;
    return o;
}

inline cfdg_config to_cfdg_config(const cfd::solver::compressible::SolverConfig& c, const GpuTimeOptions& o) {
    namespace sc = cfd::solver::compressible;
    cfdg_config g;
    cfdg_config_default(&g);
    g.viscous = c.flow_model == sc::FlowModel::ViscousFlow ? 1 : 0;
    g.gradient = c.gradient == cfd::numerics::gradient::GradientType::LeastSquaresCellFace ? CFDG_GRAD_LSQ_FACE
                                                                                           : CFDG_GRAD_LSQ_NODE;
    g.reconstruction = c.reconstruction == sc::ReconType::Muscl ? CFDG_RECON_MUSCL : CFDG_RECON_FIRST_ORDER;
    g.limiter = c.limiter == sc::LimiterType::BarthJespersen ? CFDG_LIM_BARTH_JESPERSEN
                : c.limiter == sc::LimiterType::VanAlbada  ? CFDG_LIM_VAN_ALBADA
                                                           : CFDG_LIM_VENKATAKRISHNAN;
    g.precision = o.precision;
    g.precond = c.linear_solver_params.precond_type == linalg::PreconditionerType::SGS ? CFDG_PC_SGS : CFDG_PC_NONE;
    g.sgs_ordering = o.sgs_ordering;
    g.lin_max_iterations = c.linear_solver_params.max_iterations;
    g.lin_rel_tol = c.linear_solver_params.relative_tolerance;
    g.lin_abs_tol = c.linear_solver_params.absolute_tolerance;
    g.jacobian = o.jacobian;
    g.gamma = c.flow.gamma;
    g.gas_constant = c.flow.gas_constant;
    g.prandtl = c.prandtl;
    g.init_rho = c.init_rho;
    g.init_p = c.init_p;
    for (int k = 0; k < 3; ++k) g.init_velocity[k] = c.init_velocity[k];
    g.venkat_k = c.limiter_venkat_k;
    g.cfl = g.cfl_max = c.cfl;
    g.residual_tolerance = c.residual_tolerance;
    g.max_iterations = c.max_iterations;
    return g;
}

inline std::vector<cfdg_bc_desc> to_cfdg_bcs(const cfd::bc::BoundaryConfig& b) {
    std::vector<cfdg_bc_desc> out;
    for (const auto& d : b.patches) {
        cfdg_bc_desc e{};
        e.patch_id = d.patch_id;
        e.type = static_cast<int32_t>(d.type);
        e.inflow_mode = static_cast<int32_t>(d.inflow_mode);
        e.p = d.p;
        e.t = d.t;
        e.tmp_grad = d.tmp_grad;
        for (int k = 0; k < 3; ++k) {
            e.velocity[k] = d.velocity[k];
            e.direction[k] = d.direction[k];
        }
        e.mach = d.mach;
        e.alpha_deg = d.alpha_deg;
        e.beta_deg = d.beta_deg;
        out.push_back(e);
    }
    return out;
}

// Backward Euler with the whole iteration on the GPU: advance() uploads the
// operator's state, runs cfdg_newton_step at the operator's CFL (residual,
// Jacobian, BiCGSTAB + SGS, update) and writes the new state into the stage
// slots and R(U) of the old state into the residual slots, so the Solver's
// own convergence monitor and output see what BackwardEuler leaves there.
template <typename Op>
class GpuBackwardEuler {
public:
    using Operator = Op;
    static constexpr bool kNeedsMatrix = false;  // the device holds its own matrix
    static constexpr mesh::AuxConnType kAuxConnectivity = mesh::AuxConnType::None;
    static constexpr mesh::AuxGeomType kAuxGeometry = mesh::AuxGeomType::None;
    static constexpr const char* name() noexcept { return "BACKWARD_EULER (cfdg, GPU)"; }
    static_assert(!Op::kHasModules, "GpuBackwardEuler: the mean-flow variables only");

    GpuBackwardEuler() = default;
    GpuBackwardEuler(const GpuBackwardEuler&) = delete;
    GpuBackwardEuler& operator=(const GpuBackwardEuler&) = delete;
    ~GpuBackwardEuler() { cfdg_solver_destroy(s_); }

    void advance(Op& op) noexcept {
        const MPI_Comm comm = op.mpi_comm();
        if (!s_) create(op);
        const auto u = op.u_slots();
        for (std::size_t v = 0; v < 5; ++v) std::copy(u[v], u[v] + n_, host_.begin() + v * n_);
        require(cfdg_solver_set_state(s_, host_.data(), static_cast<int64_t>(n_)), comm, "GpuBackwardEuler");
        cfdg_step_result r{};
        require(cfdg_newton_step(s_, op.config().cfl, &r), comm, "GpuBackwardEuler::advance");
        require(cfdg_solver_get_field(s_, CFDG_FIELD_RES, host_.data(), static_cast<int64_t>(5 * n_)), comm,
                "GpuBackwardEuler");
        const auto res = op.res_slots();
        for (std::size_t v = 0; v < 5; ++v) std::copy(host_.begin() + v * n_, host_.begin() + (v + 1) * n_, res[v]);
        require(cfdg_solver_get_field(s_, CFDG_FIELD_U, host_.data(), static_cast<int64_t>(5 * n_)), comm,
                "GpuBackwardEuler");
        const auto stage = op.stage_slots();
        for (std::size_t v = 0; v < 5; ++v) std::copy(host_.begin() + v * n_, host_.begin() + (v + 1) * n_, stage[v]);
        last_ = r;
        op.post_stage(op.stage_slots());
        op.ping_pong();
    }
    const cfdg_step_result& last_step() const { return last_; }

private:
    void create(Op& op) {
        const GpuTimeOptions& o = gpu_time_options();
        const MPI_Comm comm = op.mpi_comm();
        linalg::check(o.boundaries != nullptr, comm,
                      "GpuBackwardEuler: set gpu_time_options().boundaries before building the Solver");
        const MeshView view(op.mesh());
        const cfdg_config cfg = to_cfdg_config(op.config(), o);
        const std::vector<cfdg_bc_desc> bcs = to_cfdg_bcs(*o.boundaries);
        require(cfdg_solver_create(o.device, &view.v, &cfg, bcs.data(), static_cast<int32_t>(bcs.size()), &s_), comm,
                "GpuBackwardEuler: solver creation");
        n_ = static_cast<std::size_t>(op.mesh().n_own);
        host_.assign(5 * n_, 0.0);
    }
    cfdg_solver* s_ = nullptr;
    std::size_t n_ = 0;
    std::vector<double> host_;
    cfdg_step_result last_{};
};

}  // namespace cfdg::refbind
