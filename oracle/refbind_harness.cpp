// Test harness of the reference-side adapters
// (distributed-cfd-solver_b200/refbind/cfdg_reference_adapters.hpp): the
// reference's own BiCGSTAB, GradientManager-style gradient calls and
// Solver<...> iteration loop, run once with the reference's CPU classes and
// once with the GPU adapters plugged into the same seams, so the tests can
// compare the two.  Test infrastructure: compiled against the reference
// sources in place (REF_DIR) into oracle/_ref/librefbind.so, which links the
// reference build (libcfdref.so) and the product library (libcfdg.so).
#include <mpi.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "cfd/linalg/bicgstab.hpp"
#include "cfd/linalg/bsr_matrix.hpp"
#include "cfd/linalg/preconditioners.hpp"
#include "cfd/mesh/aux_connectivity.hpp"
#include "cfd/numerics/gradient/gradient_manager.hpp"
#include "cfd/numerics/limiter/slope_limiters.hpp"
#include "cfd/numerics/reconstruction/first_order.hpp"
#include "cfd/numerics/reconstruction/muscl.hpp"
#include "cfd/solver/compressible/eos/ideal_gas.hpp"
#include "cfd/solver/compressible/fluxes/hllc.hpp"
#include "cfd/solver/compressible/physics/inviscid_flow.hpp"
#include "cfd/solver/compressible/physics/stack.hpp"
#include "cfd/solver/compressible/physics/viscous_flow.hpp"
#include "cfd/solver/compressible/solver.hpp"
#include "cfd/solver/compressible/time/implicit_euler.hpp"
#include "cfd/solver/time_mode.hpp"
#include "cfdg.h"
#include "cfdg_reference_adapters.hpp"

using namespace cfd;
namespace sc = cfd::solver::compressible;
namespace rb = cfdg::refbind;

// from ref_harness.cpp
namespace refh {
mesh::MeshPart build_meshpart(const cfdg_mesh_host& v, bool with_geometry);
bc::BoundaryConfig build_bcfg(const cfdg_bc_desc* bcs, int n);
sc::SolverConfig build_cfg(const cfdg_config& c);
}  // namespace refh

#define RB_API extern "C" __attribute__((visibility("default")))

namespace {

std::unique_ptr<linalg::BsrMatrix> make_bsr(int n, int bs, const int32_t* row_ptr, const int32_t* cols,
                                            const double* vals) {
    std::vector<LocalIndex> off(n + 1, 0), val;
    for (int i = 0; i < n; ++i) {
        for (int32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
            if (cols[k] != i) val.push_back(cols[k]);
        off[i + 1] = static_cast<LocalIndex>(val.size());
    }
    auto A = std::make_unique<linalg::BsrMatrix>(MPI_COMM_WORLD, n, n, bs);
    A->assemble({}, off, val);
    std::copy(vals, vals + static_cast<std::size_t>(row_ptr[n]) * bs * bs, A->valuesData());
    return A;
}

template <typename Phys, template <typename> class Time>
using SolverOf = sc::Solver<sc::eos::IdealGas, sc::fluxes::HllcFlux,
                            numerics::recon::Muscl<numerics::limiter::Venkatakrishnan>,
                            sc::physics::PhysicsStack<Phys>, Time, solver::SteadyMode>;

// Solver::run (init_fields + run_steady: max_iterations iterations at the
// configured CFL), then the state.
template <typename Phys, template <typename> class Time>
void run_solver(const cfdg_mesh_host& m, const cfdg_config& c, const cfdg_bc_desc* bcs, int nbc, double* U_out) {
    const mesh::MeshPart mp = refh::build_meshpart(m, true);
    const sc::SolverConfig cfg = refh::build_cfg(c);
    const bc::BoundaryConfig bcfg = refh::build_bcfg(bcs, nbc);
    rb::gpu_time_options().boundaries = &bcfg;
    rb::gpu_time_options().jacobian = c.jacobian;
    rb::gpu_time_options().sgs_ordering = c.sgs_ordering;
    rb::gpu_time_options().precision = c.precision;
    const sc::eos::IdealGas eos = cfg.flow.create_ideal_gas();
    sc::physics::PhysicsStack<Phys> phys;
    if constexpr (Phys::kHasViscous) phys.base.prandtl = cfg.prandtl;
    SolverOf<Phys, Time> s(cfg, bcfg, eos, phys, mp, MPI_COMM_WORLD);
    s.run();
    const auto u = s.u_slots();
    const std::size_t n = static_cast<std::size_t>(mp.n_own);
    for (std::size_t v = 0; v < 5; ++v) std::copy(u[v], u[v] + n, U_out + v * n);
    rb::gpu_time_options().boundaries = nullptr;
}

}  // namespace

// BiCGSTAB on one BSR system through the reference's interfaces.
// mode 0: reference BiCGSTAB, reference BsrMatrix, reference SgsPreconditioner;
// mode 1: reference BiCGSTAB and BsrMatrix, GpuSgs (level sweep) set up on the BsrMatrix;
// mode 2: reference BiCGSTAB, GpuBsrOperator, GpuSgs;
// mode 3: GpuBiCGSTAB, GpuBsrOperator, GpuSgs;
// mode 4: GpuGmres(30), GpuBsrOperator, GpuSgs.
RB_API int rb_bicgstab(int n, int bs, const int32_t* row_ptr, const int32_t* cols, const double* vals,
                       const double* b, double* x, int mode, double rtol, int max_it, int* iterations, int* status,
                       double* final_residual) {
    auto A = make_bsr(n, bs, row_ptr, cols, vals);
    std::unique_ptr<rb::GpuBsrOperator> G;
    std::unique_ptr<linalg::Preconditioner> M;
    std::unique_ptr<linalg::IterativeSolver> K;
    if (mode >= 2) G = std::make_unique<rb::GpuBsrOperator>(*A);
    if (mode == 0) M = std::make_unique<linalg::SgsPreconditioner>();
    else M = std::make_unique<rb::GpuSgs>(CFDG_SGS_LEVEL);
    if (mode == 3) K = std::make_unique<rb::GpuBiCGSTAB>();
    else if (mode == 4) K = std::make_unique<rb::GpuGmres>(30);
    else K = std::make_unique<linalg::BiCGSTAB>();
    const linalg::LinearOperator& op = G ? static_cast<const linalg::LinearOperator&>(*G) : *A;
    M->setup(op);
    K->params().relative_tolerance = rtol;
    K->params().absolute_tolerance = 1e-30;
    K->params().max_iterations = max_it;
    linalg::Vector xv = A->makeVector(), bv = A->makeVector();
    std::copy(b, b + static_cast<std::size_t>(n) * bs, bv.data());
    const linalg::IterationResult r = K->solve(op, *M, xv, bv);
    std::copy(xv.data(), xv.data() + static_cast<std::size_t>(n) * bs, x);
    *iterations = r.iterations;
    *status = static_cast<int>(r.status);
    *final_residual = r.final_residual;
    return 0;
}

// GradientOperator::apply_set of nvars fields (nvars x n, cells only) with the
// reference's least-squares operator (gpu = 0) or GpuGradient (gpu = 1).
RB_API int rb_gradient(const cfdg_mesh_host* m, int stencil, int nvars, const double* q, double* g, int gpu) {
    mesh::MeshPart mp = refh::build_meshpart(*m, true);
    mesh::MeshAuxConnectivity ac;
    ac.add_connectivity(mp, mesh::AuxConnType::CellFaces | mesh::AuxConnType::CellCellsByFace);
    std::unique_ptr<numerics::gradient::GradientOperator> op;
    numerics::gradient::GradientManager gm;
    if (gpu) {
        op = std::make_unique<rb::GpuGradient>(stencil);
    } else if (stencil == CFDG_GRAD_LSQ_FACE) {
        op = std::make_unique<numerics::gradient::LeastSquaresCellFaceGradient>();
    } else {
        op = std::make_unique<numerics::gradient::LeastSquaresCellNodeGradient>();
    }
    op->setup(mp, ac);
    const std::size_t n = static_cast<std::size_t>(mp.n_cells);
    std::vector<const double*> s(nvars);
    std::vector<double*> gx(nvars), gy(nvars), gz(nvars);
    for (int v = 0; v < nvars; ++v) {
        s[v] = q + v * n;
        gx[v] = g + (3 * v + 0) * n;
        gy[v] = g + (3 * v + 1) * n;
        gz[v] = g + (3 * v + 2) * n;
    }
    op->apply_set(s, gx, gy, gz, mp, ac);
    return 0;
}

// Solver<...>::run with BackwardEuler (gpu = 0) or GpuBackwardEuler (gpu = 1)
// for c->max_iterations iterations at c->cfl; U_out gets the state (5 x n).
RB_API int rb_run(const cfdg_mesh_host* m, const cfdg_config* c, const cfdg_bc_desc* bcs, int nbc, int gpu,
                  double* U_out) {
    if (c->viscous) {
        if (gpu) run_solver<sc::physics::ViscousFlow, rb::GpuBackwardEuler>(*m, *c, bcs, nbc, U_out);
        else run_solver<sc::physics::ViscousFlow, sc::time::BackwardEuler>(*m, *c, bcs, nbc, U_out);
    } else {
        if (gpu) run_solver<sc::physics::InviscidFlow, rb::GpuBackwardEuler>(*m, *c, bcs, nbc, U_out);
        else run_solver<sc::physics::InviscidFlow, sc::time::BackwardEuler>(*m, *c, bcs, nbc, U_out);
    }
    return 0;
}
