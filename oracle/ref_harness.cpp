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
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include "cfd/linalg/bicgstab.hpp"
#include "cfd/linalg/bsr_matrix.hpp"
#include "cfd/linalg/preconditioners.hpp"
#include "cfd/mesh/aux_connectivity.hpp"
#include "cfd/mesh/aux_geometry.hpp"
#include "cfd/mesh/geometry.hpp"
#include "cfd/mesh/localmesh.hpp"
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

namespace {

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
    return s;
}

struct RefBase {
    virtual ~RefBase() = default;
    virtual void set_state(const double* U, int64_t ld) = 0;
    virtual void get_state(double* U, int64_t ld) = 0;
    virtual void stages(double* q, double* grad, double* phi, double* res, double* lam) = 0;
    virtual void jacobian(double cfl, double* alpha, double* values) = 0;
    virtual int newton_step(double cfl, double* l2, int* kit, int* kstat, double* kinit, double* kfinal) = 0;
    virtual int64_t nnzb() const = 0;
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
        time.advance(*solver);
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
                if (visc) s->impl = std::make_unique<RefImpl<sc::physics::ViscousFlow, recon::Muscl<limiter::BarthJespersen>>>(std::move(mp), cfg, bcfg, c->venkat_k);
                else s->impl = std::make_unique<RefImpl<sc::physics::InviscidFlow, recon::Muscl<limiter::BarthJespersen>>>(std::move(mp), cfg, bcfg, c->venkat_k);
                break;
            case CFDG_LIM_VAN_ALBADA:
                if (visc) s->impl = std::make_unique<RefImpl<sc::physics::ViscousFlow, recon::Muscl<limiter::VanAlbada>>>(std::move(mp), cfg, bcfg, c->venkat_k);
                else s->impl = std::make_unique<RefImpl<sc::physics::InviscidFlow, recon::Muscl<limiter::VanAlbada>>>(std::move(mp), cfg, bcfg, c->venkat_k);
                break;
            default:
                if (visc) s->impl = std::make_unique<RefImpl<sc::physics::ViscousFlow, recon::Muscl<limiter::Venkatakrishnan>>>(std::move(mp), cfg, bcfg, c->venkat_k);
                else s->impl = std::make_unique<RefImpl<sc::physics::InviscidFlow, recon::Muscl<limiter::Venkatakrishnan>>>(std::move(mp), cfg, bcfg, c->venkat_k);
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
