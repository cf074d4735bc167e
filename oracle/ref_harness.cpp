// Reference harness: a C entry layer over the reference solver's own classes,
// compiled from the reference sources in place (REF_DIR) against the
// single-rank MPI shim.  Test infrastructure only: the tests, smoke() and the
// CPU baseline of bench.py call it as the checker; the product library never
// links it.
//
// What it drives (paths inside maksim-movsisyan/Distributed-cfd-solver):
//   - mesh finalisation checks: mesh::compute_mesh_geometry (src/mesh/geometry.cpp:301),
//     mesh::validate_and_log_meshpart (src/mesh/validate.cpp:22);
//   - per-stage residual pipeline, composed from the same classes and in the
//     same order as Solver::evaluate_residual (include/cfd/solver/compressible/solver.hpp:169-247):
//     BoundaryManager, GradientManager, Muscl::compute_limiters, ResidualKernel,
//     then compute_dt (solver.hpp:256-287) and JacobianKernel (jacobian_kernel.hpp:74-103);
//   - whole nonlinear iterations through Solver<...> + time::BackwardEuler
//     (include/cfd/solver/compressible/time/implicit_euler.hpp:34-76), with the
//     CFL set per iteration through the public config();
//   - linalg: BsrMatrix, SgsPreconditioner, BiCGSTAB (src/linalg/*).
#include <mpi.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "cfd/linalg/bicgstab.hpp"
#include "cfd/linalg/bsr_matrix.hpp"
#include "cfd/linalg/preconditioners.hpp"
#include "cfd/io/vtk/vtu.hpp"
#include "cfd/mesh/aux_connectivity.hpp"
#include "cfd/mesh/aux_geometry.hpp"
#include "cfd/mesh/faces.hpp"
#include "cfd/mesh/geometry.hpp"
#include "cfd/mesh/localmesh.hpp"
#include "cfd/mesh/raw_mesh.hpp"
#include "cfd/mesh/reorder.hpp"
#include "cfd/mesh/validate.hpp"
#include "cfd/numerics/gradient/gradient_manager.hpp"
#include "cfd/numerics/limiter/slope_limiters.hpp"
#include "cfd/numerics/reconstruction/first_order.hpp"
#include "cfd/numerics/reconstruction/muscl.hpp"
#include "cfd/solver/compressible/bc_manager.hpp"
#include "cfd/solver/compressible/eos/ideal_gas.hpp"
#include "cfd/solver/compressible/fluxes/hllc.hpp"
#include "cfd/solver/compressible/jacobian_kernel.hpp"
#include "cfd/solver/compressible/physics/inviscid_flow.hpp"
#include "cfd/solver/compressible/physics/stack.hpp"
#include "cfd/solver/compressible/physics/viscous_flow.hpp"
#include "cfd/solver/compressible/residual_kernel.hpp"
#include "cfd/solver/compressible/solver.hpp"
#include "cfd/solver/compressible/time/implicit_euler.hpp"
#include "cfd/solver/time_mode.hpp"
#include "cfdg.h"

using namespace cfd;
namespace sc = cfd::solver::compressible;

#define REFH_API extern "C" __attribute__((visibility("default")))

// MeshPart / SolverConfig / BoundaryConfig from the C structures (external
// linkage: the adapter harness refbind_harness.cpp reuses them).
namespace refh {

mesh::MeshPart build_meshpart(const cfdg_mesh_host& v, bool with_geometry) {
    mesh::MeshPart mp;
    mp.rank = 0;
    mp.nprocs = 1;
    mp.n_own = mp.n_cells = v.n_cells;
    mp.n_nodes_own = mp.n_nodes = v.n_nodes;
    mp.n_faces = v.n_faces;
    mp.n_inner_faces = mp.n_internal_faces = v.n_inner_faces;
    mp.n_cells_g = v.n_cells;
    mp.n_nodes_g = v.n_nodes;
    mp.n_faces_g = v.n_faces;
    mp.n_bfaces_g = v.n_faces - v.n_inner_faces;
    const std::size_t nc = v.n_cells, nf = v.n_faces, nn = v.n_nodes;
    mp.cell_type.resize(nc);
    for (std::size_t c = 0; c < nc; ++c) mp.cell_type[c] = static_cast<mesh::CellType>(v.cell_type[c]);
    mp.cell_gid.resize(nc);
    for (std::size_t c = 0; c < nc; ++c) mp.cell_gid[c] = static_cast<GlobalIndex>(c);
    mp.cell_donor.assign(nc, -1);
    mp.cell_nodes_offsets.assign(v.cell_nodes_offsets, v.cell_nodes_offsets + nc + 1);
    mp.cell_nodes.assign(v.cell_nodes, v.cell_nodes + v.cell_nodes_offsets[nc]);
    mp.node_gid.resize(nn);
    for (std::size_t i = 0; i < nn; ++i) mp.node_gid[i] = static_cast<GlobalIndex>(i);
    mp.node_x.assign(v.node_x, v.node_x + nn);
    mp.node_y.assign(v.node_y, v.node_y + nn);
    mp.node_z.assign(v.node_z, v.node_z + nn);
    mp.face_owner.assign(v.face_owner, v.face_owner + nf);
    mp.face_neigh.assign(v.face_neigh, v.face_neigh + nf);
    mp.face_patch.assign(v.face_patch, v.face_patch + nf);
    mp.face_nodes_offsets.assign(v.face_nodes_offsets, v.face_nodes_offsets + nf + 1);
    mp.face_nodes.assign(v.face_nodes, v.face_nodes + v.face_nodes_offsets[nf]);
    mp.face_type.resize(nf);
    for (std::size_t f = 0; f < nf; ++f)
        mp.face_type[f] = (v.face_nodes_offsets[f + 1] - v.face_nodes_offsets[f] == 3) ? mesh::CellType::TRI
                                                                                        : mesh::CellType::QUAD;
    if (with_geometry) {
        mp.cell_centroid_x.assign(v.cell_centroid_x, v.cell_centroid_x + nc);
        mp.cell_centroid_y.assign(v.cell_centroid_y, v.cell_centroid_y + nc);
        mp.cell_centroid_z.assign(v.cell_centroid_z, v.cell_centroid_z + nc);
        mp.cell_volume.assign(v.cell_volume, v.cell_volume + nc);
        mp.face_centroid_x.assign(v.face_centroid_x, v.face_centroid_x + nf);
        mp.face_centroid_y.assign(v.face_centroid_y, v.face_centroid_y + nf);
        mp.face_centroid_z.assign(v.face_centroid_z, v.face_centroid_z + nf);
        mp.face_normal_x.assign(v.face_normal_x, v.face_normal_x + nf);
        mp.face_normal_y.assign(v.face_normal_y, v.face_normal_y + nf);
        mp.face_normal_z.assign(v.face_normal_z, v.face_normal_z + nf);
        mp.face_area.assign(v.face_area, v.face_area + nf);
    }
    mp.recv_offsets = {0};
    mp.send_offsets = {0};
    const int np = std::max(v.n_patches, 1);
    mp.patches.resize(np);
    for (int p = 0; p < np; ++p) {
        mp.patches[p].name = "patch" + std::to_string(p);
        mp.patches[p].cgns_type = "UserDefined";
    }
    mp.patch_face_offsets.assign(np + 1, 0);
    for (std::size_t f = 0; f < nf; ++f)
        if (mp.face_patch[f] >= 0) ++mp.patch_face_offsets[mp.face_patch[f] + 1];
    for (int p = 0; p < np; ++p) mp.patch_face_offsets[p + 1] += mp.patch_face_offsets[p];
    mp.patch_faces.resize(mp.patch_face_offsets[np]);
    std::vector<LocalIndex> cur(mp.patch_face_offsets.begin(), mp.patch_face_offsets.end() - 1);
    for (std::size_t f = 0; f < nf; ++f)
        if (mp.face_patch[f] >= 0) mp.patch_faces[cur[mp.face_patch[f]]++] = static_cast<LocalIndex>(f);
    for (int d = 0; d < 3; ++d) {
        const double* a = d == 0 ? v.node_x : (d == 1 ? v.node_y : v.node_z);
        mp.bbox_lo[d] = *std::min_element(a, a + nn);
        mp.bbox_hi[d] = *std::max_element(a, a + nn);
    }
    return mp;
}

bc::BoundaryConfig build_bcfg(const cfdg_bc_desc* bcs, int n) {
    bc::BoundaryConfig b;
    for (int i = 0; i < n; ++i) {
        bc::BCDescriptor d;
        d.type = static_cast<bc::physical::BCType>(bcs[i].type);
        d.inflow_mode = static_cast<bc::physical::InflowMode>(bcs[i].inflow_mode);
        d.patch_id = bcs[i].patch_id;
        d.p = bcs[i].p;
        d.t = bcs[i].t;
        d.tmp_grad = bcs[i].tmp_grad;
        for (int k = 0; k < 3; ++k) {
            d.velocity[k] = bcs[i].velocity[k];
            d.direction[k] = bcs[i].direction[k];
        }
        d.mach = bcs[i].mach;
        d.alpha_deg = bcs[i].alpha_deg;
        d.beta_deg = bcs[i].beta_deg;
        b.patches.push_back(d);
    }
    return b;
}

sc::SolverConfig build_cfg(const cfdg_config& c) {
    sc::SolverConfig s;
    s.flow.gamma = c.gamma;
    s.flow.gas_constant = c.gas_constant;
    s.prandtl = c.prandtl;
    s.flow_model = c.viscous ? sc::FlowModel::ViscousFlow : sc::FlowModel::InviscidFlow;
    s.init_rho = c.init_rho;
    s.init_p = c.init_p;
    for (int k = 0; k < 3; ++k) s.init_velocity[k] = c.init_velocity[k];
    s.gradient = (c.gradient == CFDG_GRAD_LSQ_FACE) ? numerics::gradient::GradientType::LeastSquaresCellFace
                                                     : numerics::gradient::GradientType::LeastSquaresCellNode;
    s.reconstruction = c.reconstruction == CFDG_RECON_MUSCL ? sc::ReconType::Muscl : sc::ReconType::FirstOrder;
    s.limiter = sc::LimiterType::Venkatakrishnan;
    s.limiter_venkat_k = c.venkat_k;
    s.scheme = sc::TimeScheme::BackwardEuler;
    s.cfl = c.cfl;
    s.max_iterations = c.max_iterations;
    s.residual_tolerance = c.residual_tolerance;
    s.time_mode = sc::TimeMode::Steady;
    s.linear_solver_params.type = linalg::SolverType::BICGSTAB;
    s.linear_solver_params.precond_type =
        c.precond == CFDG_PC_SGS ? linalg::PreconditionerType::SGS : linalg::PreconditionerType::None;
    s.linear_solver_params.relative_tolerance = c.lin_rel_tol;
    s.linear_solver_params.absolute_tolerance = c.lin_abs_tol;
    s.linear_solver_params.max_iterations = c.lin_max_iterations;
    s.linear_solver_params.verbosity = linalg::Verbosity::Silent;
    s.output_dir = "/tmp/cfdg_ref_out";
    s.field_interval = 0;
    s.residual_interval = 1;
    s.time_mode = c.time_mode == CFDG_TIME_UNSTEADY ? sc::TimeMode::Unsteady : sc::TimeMode::Steady;
    s.dt = c.dt_physical;
    s.max_time_steps = c.max_time_steps;
    s.bdf_order = c.bdf_order;
    return s;
}

}  // namespace refh

namespace {
using refh::build_bcfg;
using refh::build_cfg;
using refh::build_meshpart;

// Limiter freeze through the reference's reconstruction-policy seam
// (ReconstructionPolicy, include/cfd/numerics/reconstruction/concepts.hpp):
// while g_limiter_frozen is set, compute_limiters leaves the Solver's phi
// slots as last computed, which is what the GPU library's limiter freeze
// does.  The reference itself recomputes phi on every residual evaluation.
bool g_limiter_frozen = false;

template <typename L>
struct FreezableMuscl : numerics::recon::Muscl<L> {
    template <std::size_t NVars>
    static void compute_limiters(const mesh::MeshPart& mesh, const mesh::MeshAuxConnectivity& aux_conn,
                                 const double* const* q, const double* const* gx, const double* const* gy,
                                 const double* const* gz, double* const* phi, const double venkat_k = 1.0) noexcept {
        if (!g_limiter_frozen)
            numerics::recon::Muscl<L>::template compute_limiters<NVars>(mesh, aux_conn, q, gx, gy, gz, phi, venkat_k);
    }
};

struct RefBase {
    virtual ~RefBase() = default;
    virtual void set_state(const double* U, int64_t ld) = 0;
    virtual void get_state(double* U, int64_t ld) = 0;
    virtual void stages(double* q, double* grad, double* phi, double* res, double* lam) = 0;
    virtual void jacobian(double cfl, double* alpha, double* values) = 0;
    virtual int newton_step(double cfl, double* l2, int* kit, int* kstat, double* kinit, double* kfinal) = 0;
    virtual int64_t nnzb() const = 0;
    virtual void write_vtu(const char* outdir, const char* stem) = 0;
    bool frozen = false;
};

template <typename Phys, typename Recon>
struct RefImpl final : RefBase {
    using Stack = sc::physics::PhysicsStack<Phys>;
    using SolverT = sc::Solver<sc::eos::IdealGas, sc::fluxes::HllcFlux, Recon, Stack, sc::time::BackwardEuler,
                               solver::SteadyMode>;
    static constexpr bool kGrad = Recon::kNeedsGradients || Phys::kNeedsGradients;

    mesh::MeshPart mp;
    sc::SolverConfig cfg;
    bc::BoundaryConfig bcfg;
    sc::eos::IdealGas eos;
    Stack phys;
    mesh::MeshAuxConnectivity aux_conn;
    mesh::MeshAuxGeometry aux_geom;
    numerics::gradient::GradientManager gm;
    sc::BoundaryManager<sc::eos::IdealGas> bcs;
    std::unique_ptr<sc::ResidualKernel<sc::eos::IdealGas, sc::fluxes::HllcFlux, Recon, Stack>> rk;
    std::unique_ptr<sc::JacobianKernel<sc::eos::IdealGas, sc::fluxes::HllcFlux, Stack>> jk;
    std::unique_ptr<linalg::BsrMatrix> mat;
    std::size_t n, nt;
    std::vector<double> U, q, grad, phi, res, lam;
    // whole-iteration path
    std::unique_ptr<SolverT> solver;
    sc::time::BackwardEuler<SolverT> time;
    mesh::MeshAuxConnectivity be_conn;

    RefImpl(mesh::MeshPart&& m, const sc::SolverConfig& c, const bc::BoundaryConfig& b, double venkat)
        : mp(std::move(m)), cfg(c), bcfg(b) {
        (void)venkat;
        eos = cfg.flow.create_ideal_gas();
        if constexpr (Phys::kHasViscous) phys.base.prandtl = cfg.prandtl;
        aux_conn.add_connectivity(mp, Recon::kAuxConnectivity | Stack::kAuxConnectivity |
                                          mesh::AuxConnType::CellCellsByFace);
        aux_geom.add_geometry(mp, Recon::kAuxGeometry | Stack::kAuxGeometry);
        if constexpr (kGrad) {
            gm.create_gradient(cfg.gradient);
            gm.setup_gradient(mp, aux_conn);
        }
        bcs.initialize(bcfg, mp, eos);
        rk = std::make_unique<sc::ResidualKernel<sc::eos::IdealGas, sc::fluxes::HllcFlux, Recon, Stack>>(
            mp, aux_conn, aux_geom, eos, phys);
        jk = std::make_unique<sc::JacobianKernel<sc::eos::IdealGas, sc::fluxes::HllcFlux, Stack>>(mp, aux_conn,
                                                                                                   aux_geom, eos, phys);
        n = static_cast<std::size_t>(mp.n_cells);
        nt = n + static_cast<std::size_t>(mp.n_faces - mp.n_inner_faces);
        U.assign(5 * nt, 0.0);
        q.assign(5 * nt, 0.0);
        grad.assign(15 * nt, 0.0);
        phi.assign(5 * nt, 0.0);
        res.assign(5 * nt, 0.0);
        lam.assign(n, 0.0);
        mat = std::make_unique<linalg::BsrMatrix>(MPI_COMM_WORLD, mp.n_cells_g, mp.n_own, 5);
        mat->assemble({}, aux_conn.cell_cells_face_offsets, aux_conn.cell_cells_face);
        solver = std::make_unique<SolverT>(cfg, bcfg, eos, phys, mp, MPI_COMM_WORLD);
        be_conn.add_connectivity(mp, mesh::AuxConnType::CellCellsByFace);
        time.system_setup(mp, be_conn, cfg.linear_solver_params, MPI_COMM_WORLD);
    }

    int64_t nnzb() const override { return static_cast<int64_t>(mat->rowPtr()[n]); }

    // Solver::write_fields (solver.hpp:856-898; private there): the same
    // fields from the Solver's state through the reference's EOS helpers,
    // written by the reference's io::vtk::write_solution_vtu.
    void write_vtu(const char* outdir, const char* stem) override {
        auto u = solver->u_slots();
        std::vector<double> rho(n), vx(n), vy(n), vz(n), pr(n), mach(n);
        for (std::size_t c = 0; c < n; ++c) {
            const double U5[5] = {u[0][c], u[1][c], u[2][c], u[3][c], u[4][c]};
            const double r = U5[0];
            const double p = sc::eos::pressure(eos, U5);
            const double a = eos.sound_speed_rhop(r, p);
            rho[c] = r;
            vx[c] = U5[1] / r;
            vy[c] = U5[2] / r;
            vz[c] = U5[3] / r;
            pr[c] = p;
            mach[c] = std::sqrt(U5[1] * U5[1] + U5[2] * U5[2] + U5[3] * U5[3]) / (r * a);
        }
        const io::vtk::SolutionField f[] = {{"rho", rho.data()}, {"u", vx.data()},        {"v", vy.data()},
                                            {"w", vz.data()},     {"pressure", pr.data()}, {"mach", mach.data()}};
        io::vtk::write_solution_vtu(mp, f, 6, outdir, stem, MPI_COMM_WORLD);
    }

    void set_state(const double* Uin, int64_t ld) override {
        for (int v = 0; v < 5; ++v) {
            std::copy(Uin + v * ld, Uin + v * ld + n, U.begin() + v * nt);
            auto slots = solver->u_slots();
            std::copy(Uin + v * ld, Uin + v * ld + n, slots[v]);
        }
    }
    void get_state(double* Uout, int64_t ld) override {
        auto slots = solver->u_slots();
        for (int v = 0; v < 5; ++v) std::copy(slots[v], slots[v] + n, Uout + v * ld);
    }

    std::vector<double*> ptrs(std::vector<double>& a, std::size_t stride, int k) {
        std::vector<double*> p(k);
        for (int i = 0; i < k; ++i) p[i] = a.data() + i * stride;
        return p;
    }

    // Solver::evaluate_residual steps 1-6 on the harness-owned fields.
    void stages(double* q_out, double* grad_out, double* phi_out, double* res_out, double* lam_out) override {
        for (std::size_t c = 0; c < n; ++c) {
            const double Uc[5] = {U[c], U[nt + c], U[2 * nt + c], U[3 * nt + c], U[4 * nt + c]};
            sc::eos::conserved_to_primitives_pT(eos, Uc, q[c], q[nt + c], q[2 * nt + c], q[3 * nt + c], q[4 * nt + c]);
        }
        auto qs = ptrs(q, nt, 5);
        bcs.update_ghost_cells(qs, mp);
        std::vector<const double*> qc(qs.begin(), qs.end());
        std::vector<double*> gx(5), gy(5), gz(5), ph = ptrs(phi, nt, 5), rs = ptrs(res, nt, 5);
        for (int v = 0; v < 5; ++v) {
            gx[v] = grad.data() + (3 * v + 0) * nt;
            gy[v] = grad.data() + (3 * v + 1) * nt;
            gz[v] = grad.data() + (3 * v + 2) * nt;
        }
        std::vector<const double*> gxc(gx.begin(), gx.end()), gyc(gy.begin(), gy.end()), gzc(gz.begin(), gz.end()),
            phc(ph.begin(), ph.end());
        if constexpr (kGrad) {
            gm.apply_gradient_set(qc, gx, gy, gz, mp, aux_conn);
            bcs.update_ghost_cells_grad(qc, gx, gy, gz, mp);
            if constexpr (Recon::kNeedsGradients) {
                Recon::template compute_limiters<5>(mp, aux_conn, qc.data(), gxc.data(), gyc.data(), gzc.data(),
                                                    ph.data(), cfg.limiter_venkat_k);
            }
        }
        rk->apply(qc, gxc, gyc, gzc, phc, rs, lam.data(), nullptr, nullptr);
        if (q_out) std::copy(q.begin(), q.end(), q_out);
        if (grad_out) std::copy(grad.begin(), grad.end(), grad_out);
        if (phi_out)
            for (int v = 0; v < 5; ++v) std::copy(phi.begin() + v * nt, phi.begin() + v * nt + n, phi_out + v * n);
        if (res_out)
            for (int v = 0; v < 5; ++v) std::copy(res.begin() + v * nt, res.begin() + v * nt + n, res_out + v * n);
        if (lam_out) std::copy(lam.begin(), lam.end(), lam_out);
    }

    // compute_dt (solver.hpp:256-287) + JacobianKernel::apply after stages().
    void jacobian(double cfl, double* alpha_out, double* values_out) override {
        std::vector<double> alpha(n);
        const double inv_cfl = 1.0 / cfl;
        for (std::size_t c = 0; c < n; ++c) {
            const double l = std::max(lam[c], constants::kSpectralRadiusFloor);
            alpha[c] = (l * inv_cfl) + (mp.cell_volume[c] * 0.0);
        }
        auto qs = ptrs(q, nt, 5);
        std::vector<const double*> qc(qs.begin(), qs.end());
        jk->apply(qc, mat->rowPtr().data(), mat->cols().data(), mat->diagIndex().data(), mat->valuesData(),
                  alpha.data(), nullptr);
        if (alpha_out) std::copy(alpha.begin(), alpha.end(), alpha_out);
        if (values_out) std::copy(mat->values().begin(), mat->values().end(), values_out);
    }

    // One BackwardEuler::advance through the reference Solver.
    int newton_step(double cfl, double* l2, int* kit, int* kstat, double* kinit, double* kfinal) override {
        const_cast<sc::SolverConfig&>(solver->config()).cfl = cfl;
        g_limiter_frozen = frozen;
        time.advance(*solver);
        g_limiter_frozen = false;
        // residual_norms (solver.hpp:740-756) of the R(U) evaluated this step
        auto rs = solver->res_slots();
        for (int v = 0; v < 5; ++v) {
            double s = 0.0;
            for (std::size_t c = 0; c < n; ++c) s += rs[v][c] * rs[v][c];
            l2[v] = std::sqrt(s / static_cast<double>(std::max<std::size_t>(n, 1)));
        }
        (void)kit;
        (void)kstat;
        (void)kinit;
        (void)kfinal;
        return 0;
    }
};

}  // namespace

struct refh_solver {
    std::unique_ptr<RefBase> impl;
    int64_t n;
};

REFH_API int refh_compute_geometry(const cfdg_mesh_host* m, double* out_cell /*4*n: cx,cy,cz,vol*/,
                                   double* out_face /*7*nf: fx,fy,fz,nx,ny,nz,area*/) {
    mesh::MeshPart mp = build_meshpart(*m, false);
    mesh::compute_mesh_geometry(mp);
    const std::size_t n = mp.n_cells, nf = mp.n_faces;
    std::copy(mp.cell_centroid_x.begin(), mp.cell_centroid_x.end(), out_cell);
    std::copy(mp.cell_centroid_y.begin(), mp.cell_centroid_y.end(), out_cell + n);
    std::copy(mp.cell_centroid_z.begin(), mp.cell_centroid_z.end(), out_cell + 2 * n);
    std::copy(mp.cell_volume.begin(), mp.cell_volume.end(), out_cell + 3 * n);
    const std::vector<double>* fa[7] = {&mp.face_centroid_x, &mp.face_centroid_y, &mp.face_centroid_z,
                                        &mp.face_normal_x,   &mp.face_normal_y,   &mp.face_normal_z,
                                        &mp.face_area};
    for (int k = 0; k < 7; ++k) std::copy(fa[k]->begin(), fa[k]->end(), out_face + k * nf);
    return 0;
}

REFH_API int refh_validate(const cfdg_mesh_host* m) {
    mesh::MeshPart mp = build_meshpart(*m, true);
    mesh::validate_and_log_meshpart(mp);  // aborts through the shim on a violation
    return 0;
}

// Reference aux connectivity: kind 0 cell->faces, 1 cell->cells by face, 2 by node.
REFH_API int64_t refh_connectivity(const cfdg_mesh_host* m, int kind, int32_t* off, int32_t* val, int64_t cap) {
    mesh::MeshPart mp = build_meshpart(*m, true);
    mesh::MeshAuxConnectivity ac;
    const mesh::AuxConnType t = kind == 0 ? mesh::AuxConnType::CellFaces
                                          : (kind == 1 ? mesh::AuxConnType::CellCellsByFace
                                                       : mesh::AuxConnType::CellCellsByNode);
    ac.add_connectivity(mp, t);
    const auto& o = kind == 0 ? ac.cell_faces_offsets : (kind == 1 ? ac.cell_cells_face_offsets : ac.cell_cells_node_offsets);
    const auto& v = kind == 0 ? ac.cell_faces : (kind == 1 ? ac.cell_cells_face : ac.cell_cells_node);
    if (off) std::copy(o.begin(), o.end(), off);
    if (val && static_cast<int64_t>(v.size()) <= cap) std::copy(v.begin(), v.end(), val);
    return static_cast<int64_t>(v.size());
}

// Reference wall distance (MeshAuxGeometry::add_wall_distance,
// src/mesh/aux_geometry.cpp:609-696) over the face-neighbour stencil;
// wall[p] != 0 marks patch p as a wall.
REFH_API int refh_wall_distance(const cfdg_mesh_host* m, const uint8_t* wall, int n_patches, int max_sweeps,
                                double rel_tol, double* out) {
    mesh::MeshPart mp = build_meshpart(*m, true);
    mesh::MeshAuxConnectivity ac;
    mesh::MeshAuxGeometry ag;
    std::vector<bool> wp(static_cast<std::size_t>(n_patches));
    for (int p = 0; p < n_patches; ++p) wp[p] = wall[p] != 0;
    ag.add_wall_distance(mp, ac, MPI_COMM_WORLD, wp, mesh::WallDistStencil::FaceNeighbors, max_sweeps, rel_tol);
    std::copy(ag.cell_wall_dist.begin(), ag.cell_wall_dist.begin() + mp.n_cells, out);
    return 0;
}

REFH_API int refh_create(const cfdg_mesh_host* m, const cfdg_config* c, const cfdg_bc_desc* bcs, int nbc,
                         refh_solver** out) {
    mesh::MeshPart mp = build_meshpart(*m, true);
    const sc::SolverConfig cfg = build_cfg(*c);
    const bc::BoundaryConfig bcfg = build_bcfg(bcs, nbc);
    auto* s = new refh_solver();
    s->n = m->n_cells;
    using namespace cfd::numerics;
    const bool visc = c->viscous != 0;
    if (c->reconstruction == CFDG_RECON_MUSCL) {
        switch (c->limiter) {
            case CFDG_LIM_BARTH_JESPERSEN:
                if (visc) s->impl = std::make_unique<RefImpl<sc::physics::ViscousFlow, FreezableMuscl<limiter::BarthJespersen>>>(std::move(mp), cfg, bcfg, c->venkat_k);
                else s->impl = std::make_unique<RefImpl<sc::physics::InviscidFlow, FreezableMuscl<limiter::BarthJespersen>>>(std::move(mp), cfg, bcfg, c->venkat_k);
                break;
            case CFDG_LIM_VAN_ALBADA:
                if (visc) s->impl = std::make_unique<RefImpl<sc::physics::ViscousFlow, FreezableMuscl<limiter::VanAlbada>>>(std::move(mp), cfg, bcfg, c->venkat_k);
                else s->impl = std::make_unique<RefImpl<sc::physics::InviscidFlow, FreezableMuscl<limiter::VanAlbada>>>(std::move(mp), cfg, bcfg, c->venkat_k);
                break;
            default:
                if (visc) s->impl = std::make_unique<RefImpl<sc::physics::ViscousFlow, FreezableMuscl<limiter::Venkatakrishnan>>>(std::move(mp), cfg, bcfg, c->venkat_k);
                else s->impl = std::make_unique<RefImpl<sc::physics::InviscidFlow, FreezableMuscl<limiter::Venkatakrishnan>>>(std::move(mp), cfg, bcfg, c->venkat_k);
                break;
        }
    } else {
        if (visc) s->impl = std::make_unique<RefImpl<sc::physics::ViscousFlow, recon::FirstOrder>>(std::move(mp), cfg, bcfg, c->venkat_k);
        else s->impl = std::make_unique<RefImpl<sc::physics::InviscidFlow, recon::FirstOrder>>(std::move(mp), cfg, bcfg, c->venkat_k);
    }
    *out = s;
    return 0;
}

REFH_API void refh_destroy(refh_solver* s) { delete s; }
REFH_API int64_t refh_nnzb(refh_solver* s) { return s->impl->nnzb(); }
REFH_API int refh_write_vtu(refh_solver* s, const char* outdir, const char* stem) {
    s->impl->write_vtu(outdir, stem);
    return 0;
}
REFH_API int refh_set_state(refh_solver* s, const double* U, int64_t ld) {
    s->impl->set_state(U, ld);
    return 0;
}
REFH_API int refh_get_state(refh_solver* s, double* U, int64_t ld) {
    s->impl->get_state(U, ld);
    return 0;
}
REFH_API int refh_stages(refh_solver* s, double* q, double* grad, double* phi, double* res, double* lam) {
    s->impl->stages(q, grad, phi, res, lam);
    return 0;
}
REFH_API int refh_jacobian(refh_solver* s, double cfl, double* alpha, double* values) {
    s->impl->jacobian(cfl, alpha, values);
    return 0;
}
// Freezes (1) or releases (0) the limiter of the whole-iteration path.
REFH_API int refh_freeze_limiter(refh_solver* s, int frozen) {
    s->impl->frozen = frozen != 0;
    return 0;
}
REFH_API int refh_newton_step(refh_solver* s, double cfl, double* l2) {
    return s->impl->newton_step(cfl, l2, nullptr, nullptr, nullptr, nullptr);
}

// ------------------------------------------------------------------ linalg
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
    const std::size_t nv = static_cast<std::size_t>(row_ptr[n]) * bs * bs;
    std::copy(vals, vals + nv, A->valuesData());
    return A;
}
}  // namespace

REFH_API int refh_bsr_spmv(int n, int bs, const int32_t* row_ptr, const int32_t* cols, const double* vals,
                           const double* x, double* y, double alpha, double beta) {
    auto A = make_bsr(n, bs, row_ptr, cols, vals);
    linalg::Vector xv = A->makeVector(), yv = A->makeVector();
    std::copy(x, x + static_cast<std::size_t>(n) * bs, xv.data());
    std::copy(y, y + static_cast<std::size_t>(n) * bs, yv.data());
    A->apply(xv, yv, alpha, beta);
    std::copy(yv.data(), yv.data() + static_cast<std::size_t>(n) * bs, y);
    return 0;
}

REFH_API int refh_sgs_apply(int n, int bs, const int32_t* row_ptr, const int32_t* cols, const double* vals,
                            const double* r, double* z, int sweeps) {
    auto A = make_bsr(n, bs, row_ptr, cols, vals);
    linalg::SgsPreconditioner M;
    M.setSweeps(sweeps);
    M.setup(*A);
    linalg::Vector rv = A->makeVector(), zv = A->makeVector();
    std::copy(r, r + static_cast<std::size_t>(n) * bs, rv.data());
    M.apply(rv, zv);
    std::copy(zv.data(), zv.data() + static_cast<std::size_t>(n) * bs, z);
    return 0;
}

REFH_API int refh_bicgstab(int n, int bs, const int32_t* row_ptr, const int32_t* cols, const double* vals,
                           int precond, double rtol, double atol, int max_it, double* x, const double* b,
                           int* iterations, int* status, double* r_init, double* r_final) {
    auto A = make_bsr(n, bs, row_ptr, cols, vals);
    linalg::BiCGSTAB solver;
    solver.params().relative_tolerance = rtol;
    solver.params().absolute_tolerance = atol;
    solver.params().max_iterations = max_it;
    std::unique_ptr<linalg::Preconditioner> M;
    if (precond == CFDG_PC_SGS) M = std::make_unique<linalg::SgsPreconditioner>();
    else M = std::make_unique<linalg::IdentityPreconditioner>();
    M->setup(*A);
    linalg::Vector xv = A->makeVector(), bv = A->makeVector();
    std::copy(x, x + static_cast<std::size_t>(n) * bs, xv.data());
    std::copy(b, b + static_cast<std::size_t>(n) * bs, bv.data());
    const linalg::IterationResult r = solver.solve(*A, *M, xv, bv);
    std::copy(xv.data(), xv.data() + static_cast<std::size_t>(n) * bs, x);
    *iterations = r.iterations;
    *status = static_cast<int>(r.status);
    *r_init = r.initial_residual;
    *r_final = r.final_residual;
    return 0;
}

// ------------------------------------------------------------------ meshes
// The benchmark meshes built through the reference's own preprocessing
// pipeline, as apps/mesh_partition.cpp:198-405 runs it at one rank:
// RawMesh (cells with CGNS node order, node coordinates, boundary surface
// elements with their patch) -> mesh::build_faces (src/mesh/faces.cpp) ->
// mesh::migrate_local_mesh with every cell on rank 0 (src/mesh/localmesh.cpp)
// -> compute_mesh_geometry -> reorder_local_mesh(RCM) -> validate.
// The node coordinates, cell connectivity, boundary patches and the seeded
// cell shuffle restate the synthetic generator of the benchmark cases
// (cfdg_mesh_spec: structured block, plate stretching with a cap, ramp and
// circular-arc bump walls, seeded node jitter, Kuhn split into tetrahedra);
// faces, their order, geometry and the RCM numbering are the reference's.
namespace {

struct Mt64 {
    std::mt19937_64 g;
    explicit Mt64(uint64_t s) : g(s) {}
    double sym() { return 2.0 * (static_cast<double>(g() >> 11) * (1.0 / 9007199254740992.0)) - 1.0; }
};

struct RawGen {
    std::vector<double> x, y, z;
    std::vector<uint8_t> type;
    std::vector<int32_t> off, nodes;
    std::vector<std::array<int32_t, 4>> bface;  // boundary face nodes (-1 padded)
    std::vector<int32_t> bpatch;
    int n_patches = 0;
};

RawGen generate_raw(const cfdg_mesh_spec& s) {
    RawGen r;
    const int64_t NX = s.nx + 1, NY = s.ny + 1, NZ = s.nz + 1;
    auto nid = [&](int64_t i, int64_t j, int64_t k) { return static_cast<int32_t>((k * NY + j) * NX + i); };
    std::vector<double> xs(NX), ys(NY), zs(NZ);
    for (int64_t i = 0; i < NX; ++i) xs[i] = s.lx * double(i) / double(s.nx);
    for (int64_t k = 0; k < NZ; ++k) zs[k] = s.lz * double(k) / double(s.nz);
    if (s.kind == 1) {
        ys[0] = 0.0;
        double h = s.first_spacing > 0 ? s.first_spacing : s.ly / s.ny;
        for (int64_t j = 1; j < NY; ++j) {
            ys[j] = ys[j - 1] + h;
            double hn = h * (s.stretch > 0 ? s.stretch : 1.0);
            if (s.cap_spacing > 0 && hn > s.cap_spacing) hn = s.cap_spacing;
            h = hn;
        }
    } else {
        for (int64_t j = 0; j < NY; ++j) ys[j] = s.ly * double(j) / double(s.ny);
    }
    auto wall = [&](double xv) {
        if (s.kind == 0) return std::max(0.0, (xv - s.ramp_x) * std::tan(s.ramp_angle_deg * M_PI / 180.0));
        if (s.kind == 2 && s.bump_height > 0 && xv > s.bump_x0 && xv < s.bump_x1) {
            const double half = 0.5 * (s.bump_x1 - s.bump_x0), hh = s.bump_height * (s.bump_x1 - s.bump_x0);
            const double R = (half * half + hh * hh) / (2.0 * hh), xm = 0.5 * (s.bump_x0 + s.bump_x1);
            return std::sqrt(std::max(0.0, R * R - (xv - xm) * (xv - xm))) + (hh - R);
        }
        return 0.0;
    };
    const int64_t nn = NX * NY * NZ;
    r.x.resize(nn);
    r.y.resize(nn);
    r.z.resize(nn);
    for (int64_t k = 0; k < NZ; ++k)
        for (int64_t j = 0; j < NY; ++j)
            for (int64_t i = 0; i < NX; ++i) {
                const int32_t n = nid(i, j, k);
                r.x[n] = xs[i];
                r.y[n] = s.kind == 1 ? ys[j] : wall(xs[i]) + (ys[j] / s.ly) * (s.ly - wall(xs[i]));
                r.z[n] = zs[k];
            }
    if (s.jitter > 0) {
        Mt64 rng(s.seed ^ 0x9e3779b97f4a7c15ULL);
        const std::vector<double> x0(r.x), y0(r.y), z0(r.z);
        if (s.kind == 1) {  // whole wall-normal lines in x/z, whole rows in y
            for (int64_t k = 1; k < NZ - 1; ++k)
                for (int64_t i = 1; i < NX - 1; ++i) {
                    const double ox = s.jitter * std::min(xs[i + 1] - xs[i], xs[i] - xs[i - 1]) * rng.sym();
                    const double oz = s.jitter * std::min(zs[k + 1] - zs[k], zs[k] - zs[k - 1]) * rng.sym();
                    for (int64_t j = 0; j < NY; ++j) {
                        r.x[nid(i, j, k)] = x0[nid(i, j, k)] + ox;
                        r.z[nid(i, j, k)] = z0[nid(i, j, k)] + oz;
                    }
                }
            for (int64_t j = 1; j < NY - 1; ++j) {
                const double oy = s.jitter * std::min(ys[j + 1] - ys[j], ys[j] - ys[j - 1]) * rng.sym();
                for (int64_t k = 0; k < NZ; ++k)
                    for (int64_t i = 0; i < NX; ++i) r.y[nid(i, j, k)] = y0[nid(i, j, k)] + oy;
            }
        } else {  // every interior node by a fraction of its shortest edge
            auto d = [&](int32_t a, int32_t b) {
                return std::sqrt((x0[a] - x0[b]) * (x0[a] - x0[b]) + (y0[a] - y0[b]) * (y0[a] - y0[b]) +
                                 (z0[a] - z0[b]) * (z0[a] - z0[b]));
            };
            for (int64_t k = 1; k < NZ - 1; ++k)
                for (int64_t j = 1; j < NY - 1; ++j)
                    for (int64_t i = 1; i < NX - 1; ++i) {
                        const int32_t n = nid(i, j, k);
                        const double h = std::min({d(n, nid(i + 1, j, k)), d(n, nid(i - 1, j, k)), d(n, nid(i, j + 1, k)),
                                                   d(n, nid(i, j - 1, k)), d(n, nid(i, j, k + 1)), d(n, nid(i, j, k - 1))});
                        r.x[n] = x0[n] + s.jitter * h * rng.sym();
                        r.y[n] = y0[n] + s.jitter * h * rng.sym();
                        r.z[n] = z0[n] + s.jitter * h * rng.sym();
                    }
        }
    }
    r.off.push_back(0);
    for (int64_t k = 0; k < s.nz; ++k)
        for (int64_t j = 0; j < s.ny; ++j)
            for (int64_t i = 0; i < s.nx; ++i) {
                const int32_t v[8] = {nid(i, j, k),     nid(i + 1, j, k),     nid(i + 1, j + 1, k),     nid(i, j + 1, k),
                                      nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)};
                if (s.kind != 2) {
                    r.type.push_back(static_cast<uint8_t>(mesh::CellType::HEXA));
                    r.nodes.insert(r.nodes.end(), v, v + 8);
                    r.off.push_back(static_cast<int32_t>(r.nodes.size()));
                    continue;
                }
                // six tetrahedra around the (0,0,0)-(1,1,1) diagonal, one per
                // axis order; corners listed so that det[n1-n0,n2-n0,n3-n0] > 0
                static const int ord[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
                for (const auto& o : ord) {
                    int bits = 0, corner[4] = {0, 0, 0, 0};
                    for (int q = 0; q < 3; ++q) corner[q + 1] = (bits |= 1 << o[q]);
                    int32_t t[4];
                    for (int q = 0; q < 4; ++q)
                        t[q] = nid(i + (corner[q] & 1), j + ((corner[q] >> 1) & 1), k + ((corner[q] >> 2) & 1));
                    double e[3][3];
                    for (int q = 0; q < 3; ++q) {
                        e[q][0] = r.x[t[q + 1]] - r.x[t[0]];
                        e[q][1] = r.y[t[q + 1]] - r.y[t[0]];
                        e[q][2] = r.z[t[q + 1]] - r.z[t[0]];
                    }
                    const double det = e[0][0] * (e[1][1] * e[2][2] - e[1][2] * e[2][1]) -
                                       e[0][1] * (e[1][0] * e[2][2] - e[1][2] * e[2][0]) +
                                       e[0][2] * (e[1][0] * e[2][1] - e[1][1] * e[2][0]);
                    if (det < 0) std::swap(t[1], t[2]);
                    r.type.push_back(static_cast<uint8_t>(mesh::CellType::TET));
                    r.nodes.insert(r.nodes.end(), t, t + 4);
                    r.off.push_back(static_cast<int32_t>(r.nodes.size()));
                }
            }
    // boundary surface elements: cell faces whose nodes all lie on one
    // boundary plane; patches ramp/bump 0 inlet 1 outlet 2 top 3 wall
    // 4 z-planes; plate additionally 5 = lower symmetry ahead of plate_x0
    r.n_patches = s.kind == 1 ? 6 : 5;
    const std::size_t nc = r.type.size();
    for (std::size_t c = 0; c < nc; ++c) {
        const int ti = r.type[c];
        for (int f = 0; f < mesh::kFacesPerType[ti]; ++f) {
            const int fn = mesh::kFaceNodes[ti][f];
            std::array<int32_t, 4> fnodes = {-1, -1, -1, -1};
            bool i0 = true, iN = true, j0 = true, jN = true, k0 = true, kN = true;
            double xc = 0.0;
            for (int q = 0; q < fn; ++q) {
                const int32_t n = r.nodes[r.off[c] + mesh::kFaceTable[ti][f][q]];
                fnodes[q] = n;
                const int64_t i = n % NX, j = (n / NX) % NY, k = n / (NX * NY);
                i0 &= i == 0;
                iN &= i == NX - 1;
                j0 &= j == 0;
                jN &= j == NY - 1;
                k0 &= k == 0;
                kN &= k == NZ - 1;
                xc += xs[i] / fn;
            }
            int p = -1;
            if (i0) p = 0;
            else if (iN) p = 1;
            else if (jN) p = 2;
            else if (j0) p = (s.kind == 1 && xc < s.plate_x0) ? 5 : 3;
            else if (k0 || kN) p = 4;
            if (p < 0) continue;
            r.bface.push_back(fnodes);
            r.bpatch.push_back(p);
        }
    }
    return r;
}

}  // namespace

struct refh_mesh {
    mesh::MeshPart mp;
    cfdg_mesh_host view{};
};

REFH_API int refh_mesh_generate(const cfdg_mesh_spec* spec, refh_mesh** out) {
    const cfdg_mesh_spec& s = *spec;
    if (s.nx < 1 || s.ny < 1 || s.nz < 1 || s.kind < 0 || s.kind > 2) return -1;
    RawGen g = generate_raw(s);
    const int64_t nc = static_cast<int64_t>(g.type.size()), nn = static_cast<int64_t>(g.x.size());
    // seeded shuffle of the cell numbering (Fisher-Yates), before the
    // reference's own renumbering
    std::vector<int32_t> order(nc);
    for (int64_t c = 0; c < nc; ++c) order[c] = static_cast<int32_t>(c);
    if (s.permute) {
        Mt64 rng(s.seed);
        for (int64_t i = nc - 1; i > 0; --i)
            std::swap(order[i], order[static_cast<int64_t>(rng.g() % static_cast<uint64_t>(i + 1))]);
    }
    mesh::RawMesh raw;
    raw.nprocs = 1;
    raw.rank = 0;
    raw.comm = MPI_COMM_WORLD;
    raw.n_cells_g = nc;
    raw.n_nodes_g = nn;
    raw.cell_displ = {0, static_cast<GlobalIndex>(nc)};
    raw.node_displ = {0, static_cast<GlobalIndex>(nn)};
    raw.ctype.resize(nc);
    raw.cnodes_offsets.assign(1, 0);
    for (int64_t c = 0; c < nc; ++c) {
        const int32_t o = order[c];
        raw.ctype[c] = static_cast<mesh::CellType>(g.type[o]);
        for (int32_t q = g.off[o]; q < g.off[o + 1]; ++q) raw.cnodes.push_back(g.nodes[q]);
        raw.cnodes_offsets.push_back(static_cast<LocalIndex>(raw.cnodes.size()));
    }
    raw.my_node_coords_x = std::move(g.x);
    raw.my_node_coords_y = std::move(g.y);
    raw.my_node_coords_z = std::move(g.z);
    raw.surf_elems.resize(g.bface.size());
    for (std::size_t b = 0; b < g.bface.size(); ++b) {
        mesh::SurfElem& e = raw.surf_elems[b];
        int cnt = 0;
        for (int q = 0; q < 4; ++q)
            if (g.bface[b][q] >= 0) e.key.v[cnt++] = g.bface[b][q];
        std::sort(e.key.v.begin(), e.key.v.begin() + cnt);
        e.eid = static_cast<GlobalIndex>(b + 1);
        e.patch = g.bpatch[b];
    }
    for (int p = 0; p < g.n_patches; ++p) {
        mesh::BCMeta m;
        m.name = "patch" + std::to_string(p);
        m.cgns_type = "UserDefined";
        raw.bcs.push_back(m);
        raw.patch_list.emplace_back(m.name, m.cgns_type);
    }
    mesh::BuildFacesResult bf = mesh::build_faces(raw);
    partition::PartitionResult pr;
    pr.cell_target_rank.assign(static_cast<std::size_t>(nc), 0);
    pr.part2rank = {0};
    pr.rank2part = {0};
    auto* m = new refh_mesh();
    mesh::migrate_local_mesh(std::move(raw), std::move(bf.faces), pr, m->mp);
    mesh::compute_mesh_geometry(m->mp);
    if (s.reorder_rcm) mesh::reorder_local_mesh(m->mp, mesh::ReorderMethod::RCM);
    mesh::validate_and_log_meshpart(m->mp);
    mesh::MeshPart& mp = m->mp;
    cfdg_mesh_host& v = m->view;
    v.n_cells = mp.n_cells;
    v.n_faces = mp.n_faces;
    v.n_inner_faces = mp.n_inner_faces;
    v.n_nodes = mp.n_nodes;
    v.n_patches = static_cast<int32_t>(mp.patches.size());
    v.cell_type = reinterpret_cast<const uint8_t*>(mp.cell_type.data());
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
    *out = m;
    return 0;
}

REFH_API int refh_mesh_view(const refh_mesh* m, cfdg_mesh_host* view) {
    *view = m->view;
    return 0;
}

REFH_API void refh_mesh_free(refh_mesh* m) { delete m; }

// ------------------------------------------------------------ dual time
// Solver<..., BackwardEuler, UnsteadyMode<order>>::run: init_fields, then
// run_dual_time (solver.hpp:662-736) over max_time_steps physical steps of
// dt, each with up to max_iterations sub-iterations at the configured CFL.
namespace {
template <typename Phys, int Order>
void run_unsteady_ref(const cfdg_mesh_host& m, const cfdg_config& c, const cfdg_bc_desc* bcs, int nbc,
                      double* U_out) {
    using Stack = sc::physics::PhysicsStack<Phys>;
    using SolverT = sc::Solver<sc::eos::IdealGas, sc::fluxes::HllcFlux,
                               numerics::recon::Muscl<numerics::limiter::Venkatakrishnan>, Stack,
                               sc::time::BackwardEuler, solver::UnsteadyMode<Order>>;
    const mesh::MeshPart mp = build_meshpart(m, true);
    const sc::SolverConfig cfg = build_cfg(c);
    const bc::BoundaryConfig bcfg = build_bcfg(bcs, nbc);
    const sc::eos::IdealGas eos = cfg.flow.create_ideal_gas();
    Stack phys;
    if constexpr (Phys::kHasViscous) phys.base.prandtl = cfg.prandtl;
    SolverT s(cfg, bcfg, eos, phys, mp, MPI_COMM_WORLD);
    s.run();
    const auto u = s.u_slots();
    const std::size_t n = static_cast<std::size_t>(mp.n_own);
    for (std::size_t v = 0; v < 5; ++v) std::copy(u[v], u[v] + n, U_out + v * n);
}
}  // namespace

REFH_API int refh_run_unsteady(const cfdg_mesh_host* m, const cfdg_config* c, const cfdg_bc_desc* bcs, int nbc,
                               double* U_out) {
    if (c->bdf_order == 1) {
        if (c->viscous) run_unsteady_ref<sc::physics::ViscousFlow, 1>(*m, *c, bcs, nbc, U_out);
        else run_unsteady_ref<sc::physics::InviscidFlow, 1>(*m, *c, bcs, nbc, U_out);
    } else {
        if (c->viscous) run_unsteady_ref<sc::physics::ViscousFlow, 2>(*m, *c, bcs, nbc, U_out);
        else run_unsteady_ref<sc::physics::InviscidFlow, 2>(*m, *c, bcs, nbc, U_out);
    }
    return 0;
}
