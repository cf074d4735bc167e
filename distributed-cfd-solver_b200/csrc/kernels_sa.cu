// Spalart-Allmaras one-equation model on the device: ghost values and eddy
// viscosity, the nu_tilde face sweep (upwind convection on the mean-flow
// mass flux + skew-corrected diffusion), the cell gather with production /
// destruction / cb2 sources, and per face / cell the derivatives that the
// Jacobian kernels place in the nu_tilde entries of the 6x6 Picard blocks.  Follows include/cfd/solver/compressible/turbulence/
// spalart_allmaras.hpp (the reference module, which does not compile) with
// the standard SA-1994 signs restored: the diffusive flux enters the
// residual with a minus sign, the cb2 term is a source, S = sqrt(2 S_ij S_ij)
// with full weight on the shear terms, and
// f_w = g ((1 + cw3^6) / (g^6 + cw3^6))^(1/6).  At walls and symmetry planes
// the boundary face is never treated as an inflow (the reference tests the
// sign of a mass flux that is zero up to round-off there).
#include "kernels.hpp"
#include "physics.cuh"

namespace cfdg {

namespace {

constexpr double kSbarFloor = 1.0e-10;
constexpr double kMinWallDist = 1.0e-10;

// Ghost rho*nu_tilde (SpalartAllmaras::apply_bcs, spalart_allmaras.hpp:234-257)
// and the pre-sweep (:263-282): density, nu_tilde, eddy viscosity on cells,
// zero eddy viscosity on BC ghosts.  Threads [0,n) cells, [n,n+nb) ghosts.
__global__ void k_sa_pre(DevMesh m, DevFields f, GasParams g, SaParams sa, double* __restrict__ rhonu_g) {
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t n = m.n, nt = m.nt;
    if (t < n) {
        const double rho = f.q[t] / (g.R * f.q[4 * nt + t]);
        const double nu = f.U[5 * n + t] / rho;
        f.rho[t] = rho;
        f.nu[t] = nu;
        const double nu_lam = sutherland(f.q[4 * nt + t]) / rho;
        const double chi = nu / nu_lam, chi3 = chi * chi * chi;
        const double fv1 = chi3 / (chi3 + sa.cv1 * sa.cv1 * sa.cv1);
        f.mut[t] = rho * nu * fv1;
    } else if (t < n + m.nb) {
        const int64_t b = t - n;
        const int32_t c0 = m.owner[m.ni + b];
        const int kind = m.patches[m.bpatch[b]].sa_kind;
        const double rn0 = f.U[5 * n + c0];
        double rg;
        if (kind == 0) rg = -rn0;
        else if (kind == 1) rg = (f.q[t] / (g.R * f.q[4 * nt + t])) * sa.nu_inf;
        else rg = rn0;
        rhonu_g[b] = rg;
        f.mut[t] = 0.0;
        f.rho[t] = 0.0;
        f.nu[t] = 0.0;
    }
}

// Face sweep (SpalartAllmaras::face_sweep, spalart_allmaras.hpp:291-368):
// Face-major pairs: out[2f] = convective - diffusive nu_tilde flux,
// out[2f+1] = spectral-radius increment (interior faces); jac[2f] /
// jac[2f+1] = d flux / d(rho nu_tilde) of owner / neighbour (boundary
// faces: owner incl. the ghost's dependence).  A cell's gather then reads
// one 16-byte pair per face.
__global__ void __launch_bounds__(128) k_sa_face(DevMesh m, DevFields f, GasParams g, SaParams sa,
                                                 const double* __restrict__ rhonu_g, const double* __restrict__ gnu,
                                                 double* __restrict__ out, double* __restrict__ jac) {
    const int32_t fc = blockIdx.x * blockDim.x + threadIdx.x;
    if (fc >= m.nf) return;
    const int64_t nt = m.nt, nf = m.nf;
    const bool inner = fc < m.ni;
    const int32_t c0 = m.owner[fc];
    const int64_t c1 = inner ? m.neigh[fc] : int64_t(m.n) + (fc - m.ni);
    const double nx = m.fnx[fc], ny = m.fny[fc], nz = m.fnz[fc], A = m.farea[fc];
    const double mf = f.fflux[int64_t(fc) * 6];  // mass flux of the mean-flow sweep (entry 0 of the face record)
    const double is = 1.0 / sa.sigma;
    const double dx = m.fdx[fc], dy = m.fdy[fc], dz = m.fdz[fc], id = m.finv_d[fc];
    const double nu0 = f.nu[c0];
    double nu1, rho1, sgn1 = 1.0, dg = 0.0;
    bool inflow = false;
    if (inner) {
        nu1 = f.nu[c1];
        rho1 = f.rho[c1];
    } else {
        const int64_t b = fc - m.ni;
        const int kind = m.patches[m.bpatch[b]].sa_kind;
        rho1 = f.q[c1] / (g.R * f.q[4 * nt + c1]);
        // walls and symmetry planes carry no mass flux (their mf is
        // round-off): only inflow/outflow patches switch on its sign
        inflow = (kind == 1 || kind == 2) && mf < 0.0;
        nu1 = inflow ? sa.nu_inf : rhonu_g[b] / rho1;
        sgn1 = (kind == 0) ? -1.0 : 1.0;  // ghost gradient mirrors the owner's, flipped at walls
        if (!inflow) dg = (kind == 0) ? -1.0 / rho1 : (kind == 1 ? 0.0 : 1.0 / rho1);
    }
    // averaged + skew-corrected face gradient (face_gradient, :486-508)
    double g0 = gnu[c0], g1 = gnu[nt + c0], g2 = gnu[2 * nt + c0];
    double h0, h1, h2;
    if (inner) {
        h0 = gnu[c1];
        h1 = gnu[nt + c1];
        h2 = gnu[2 * nt + c1];
    } else {
        h0 = sgn1 * g0;
        h1 = sgn1 * g1;
        h2 = sgn1 * g2;
    }
    double gn0 = 0.5 * (g0 + h0), gn1 = 0.5 * (g1 + h1), gn2 = 0.5 * (g2 + h2);
    const double gd = gn0 * dx + gn1 * dy + gn2 * dz;
    const double corr = ((nu1 - nu0) - gd) * id * id;
    gn0 += corr * dx;
    gn1 += corr * dy;
    gn2 += corr * dz;
    const double Tf = 0.5 * (f.q[4 * nt + c0] + f.q[4 * nt + c1]);
    const double mu_f = sutherland(Tf);
    const double rho0 = f.rho[c0];
    const double rho_f = 0.5 * (rho0 + rho1);
    // interior: rho_f * nu_f with nu_f the face average; boundary: the
    // reference's rho_f * 0.5 * (nu0 + nu_g) evaluation order
    const double coef = inner ? is * (mu_f + rho_f * (0.5 * (nu0 + nu1))) : is * (mu_f + rho_f * 0.5 * (nu0 + nu1));
    const double fd = coef * (gn0 * nx + gn1 * ny + gn2 * nz) * A;
    double nu_up;
    if (inner) nu_up = (mf >= 0.0) ? nu0 : nu1;
    else nu_up = inflow ? sa.nu_inf : nu0;
    const double lam_inc =
        inner ? (fabs(mf) / rho_f + 2.0 * is * (mu_f + rho_f * (0.5 * (nu0 + nu1))) / rho_f * A * id) : 0.0;
    reinterpret_cast<double2*>(out)[fc] = make_double2(mf * nu_up - fd, lam_inc);
    const double cd = coef * A * id;
    if (inner)
        reinterpret_cast<double2*>(jac)[fc] = make_double2((fmax(mf, 0.0) + cd) / rho0, (fmin(mf, 0.0) - cd) / rho1);
    else
        reinterpret_cast<double2*>(jac)[fc] = make_double2((inflow ? 0.0 : mf / rho0) + cd * (1.0 / rho0 - dg), 0.0);
}

// Cell gather of the nu_tilde fluxes (ascending face order, as the
// sequential reference), spectral radius increments, and the cell sources
// (SpalartAllmaras::cell_sources, spalart_allmaras.hpp:376-432); dsrc = the
// destruction derivative V 2 cw1 fw nu / d^2 for the Jacobian diagonal.
__global__ void __launch_bounds__(128) k_sa_cell(DevMesh m, DevFields f, SaParams sa, const double* __restrict__ face,
                                                 const double* __restrict__ gnu, double* __restrict__ dsrc) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.n) return;
    const int64_t nt = m.nt, n = m.n;
    double r = 0.0, l = f.lam[c];
    for (int32_t e = m.c2f_off[c]; e < m.c2f_off[c + 1]; ++e) {
        const int32_t es = __ldg(m.c2fs + e);  // the side is in the sign: no owner gather
        const int32_t fc = es >= 0 ? es : ~es;
        const double2 fr = __ldg(reinterpret_cast<const double2*>(face) + fc);
        if (es >= 0) r += fr.x;
        else r -= fr.x;
        if (fc < m.ni) l += fr.y;
    }
    f.lam[c] = l;
    const double rho = f.rho[c], nu = f.nu[c];
    const double d = fmax(m.wall_dist[c], kMinWallDist), id2 = 1.0 / (d * d);
    const double* gr = f.grad;
    const double ux = gr[3 * nt + c], uy = gr[4 * nt + c], uz = gr[5 * nt + c];
    const double vx = gr[6 * nt + c], vy = gr[7 * nt + c], vz = gr[8 * nt + c];
    const double wx = gr[9 * nt + c], wy = gr[10 * nt + c], wz = gr[11 * nt + c];
    const double sxy = uy + vx, sxz = uz + wx, syz = vz + wy;
    const double s2 = 2.0 * (ux * ux + vy * vy + wz * wz) + sxy * sxy + sxz * sxz + syz * syz;
    const double S = sqrt(fmax(s2, 0.0));
    const double nu_lam = sutherland(f.q[4 * nt + c]) / rho;
    const double chi = nu / nu_lam, chi3 = chi * chi * chi;
    const double fv1 = chi3 / (chi3 + sa.cv1 * sa.cv1 * sa.cv1);
    const double fv2 = 1.0 - chi / (1.0 + chi * fv1);
    const double ik2 = 1.0 / (sa.kappa * sa.kappa);
    const double sbar = fmax(S + nu * fv2 * ik2 * id2, kSbarFloor);
    double rr = nu / (sbar * sa.kappa * sa.kappa * d * d);
    rr = fmin(fmax(rr, 0.0), 10.0);
    const double r2 = rr * rr, r6 = r2 * r2 * r2;
    const double gg = rr + sa.cw2 * (r6 - rr);
    const double g2 = gg * gg, g6 = g2 * g2 * g2;
    const double cw3_2 = sa.cw3 * sa.cw3, cw3_6 = cw3_2 * cw3_2 * cw3_2;
    const double fw = gg * pow((1.0 + cw3_6) / (g6 + cw3_6), 1.0 / 6.0);
    const double P = sa.cb1 * sbar * rho * nu;
    const double D = sa.cw1 * fw * rho * nu * nu * id2;
    const double gx = gnu[c], gy = gnu[nt + c], gz = gnu[2 * nt + c];
    const double cb2 = (sa.cb2 / sa.sigma) * rho * (gx * gx + gy * gy + gz * gz);
    f.res[5 * n + c] = r + m.vol[c] * (D - P - cb2);
    dsrc[c] = m.vol[c] * 2.0 * sa.cw1 * fw * nu * id2;
}

}  // namespace

void launch_sa_pre(const DevMesh& m, const DevFields& f, const GasParams& g, const SaParams& sa, double* rhonu_g,
                   cudaStream_t s) {
    k_sa_pre<<<grid_for(int64_t(m.n) + m.nb, 256), 256, 0, s>>>(m, f, g, sa, rhonu_g);
}

void launch_sa_sweep(const DevMesh& m, const DevFields& f, const GasParams& g, const SaParams& sa,
                     const double* rhonu_g, const double* gnu, double* face, double* jac, double* dsrc,
                     cudaStream_t s) {
    k_sa_face<<<grid_for(m.nf, 128), 128, 0, s>>>(m, f, g, sa, rhonu_g, gnu, face, jac);
    k_sa_cell<<<grid_for(m.n, 128), 128, 0, s>>>(m, f, sa, face, gnu, dsrc);
}


// Solution output fields of Solver::write_fields (solver.hpp:856-898) from
// the conserved state: rho, u, v, w, pressure (eos::pressure), Mach
// (|rho u| / (rho a), a = sqrt(gamma p / rho)), and with the turbulence model
// nu_tilde and mu_t = rho nu_tilde f_v1 (SpalartAllmaras::append_output).
__global__ void k_output_fields(int32_t n, int nv, const double* __restrict__ U, GasParams g, double cv1,
                                double* __restrict__ out) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const int64_t N = n;
    const double r = U[c], ru = U[N + c], rv = U[2 * N + c], rw = U[3 * N + c], E = U[4 * N + c];
    const double inv_rho = 1.0 / r;
    const double q2 = (ru * ru + rv * rv + rw * rw) * (inv_rho * inv_rho);
    const double e = (E * inv_rho) - 0.5 * q2;
    const double p = (g.gamma - 1.0) * r * e;
    const double a = sqrt(g.gamma * p / r);
    out[c] = r;
    out[N + c] = ru / r;
    out[2 * N + c] = rv / r;
    out[3 * N + c] = rw / r;
    out[4 * N + c] = p;
    out[5 * N + c] = sqrt(ru * ru + rv * rv + rw * rw) / (r * a);
    if (nv == 6) {
        const double nu = U[5 * N + c] / r;
        const double T = p / (r * g.R);
        const double chi = nu / (sutherland(T) / r), chi3 = chi * chi * chi;
        out[6 * N + c] = nu;
        out[7 * N + c] = r * nu * (chi3 / (chi3 + cv1 * cv1 * cv1));
    }
}

void launch_output_fields(int32_t n, int nv, const double* U, const GasParams& g, double cv1, double* out,
                          cudaStream_t s) {
    if (n > 0) k_output_fields<<<grid_for(n, 256), 256, 0, s>>>(n, nv, U, g, cv1, out);
}

}  // namespace cfdg
