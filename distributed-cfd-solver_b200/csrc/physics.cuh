// Per-face and per-cell physics as device functions: ideal-gas conversions,
// HLLC flux and its Picard Jacobian, Navier-Stokes viscous flux and its
// thin-layer Jacobian, multidimensional limiters, boundary ghost rules.
// Each function states the reference routine whose arithmetic it follows
// (paths inside maksim-movsisyan/Distributed-cfd-solver).
#pragma once

#include "device_common.cuh"

namespace cfdg {

// Sutherland constants and floors (include/cfd/core/types.hpp:48-55).
constexpr double kSuthMu = 1.716e-5;
constexpr double kSuthTRef = 273.15;
constexpr double kSuthS = 110.4;
constexpr double kLamFloor = 1.0e-14;

// ---------------------------------------------------------------- EOS
// primitives_pT_to_conserved (eos/state_conversions.hpp:115-129), IdealGas.
__device__ __forceinline__ void prim_to_cons(const GasParams& g, double p, double u, double v, double w, double T,
                                             double U[5]) {
    const double rho = p / (g.R * T);
    const double e = g.cv * T;
    const double ke = 0.5 * rho * (u * u + v * v + w * w);
    U[0] = rho;
    U[1] = rho * u;
    U[2] = rho * v;
    U[3] = rho * w;
    U[4] = rho * e + ke;
}

// conserved_to_primitives_pT (eos/state_conversions.hpp:74-89).
__device__ __forceinline__ void cons_to_prim(const GasParams& g, const double U[5], double& p, double& u, double& v,
                                             double& w, double& T) {
    const double rho = U[0];
    const double inv_rho = 1.0 / rho;
    u = U[1] * inv_rho;
    v = U[2] * inv_rho;
    w = U[3] * inv_rho;
    const double q2 = u * u + v * v + w * w;
    const double e = (U[4] * inv_rho) - 0.5 * q2;
    p = (g.gamma - 1.0) * rho * e;
    T = e / g.cv;
}

// eos::pressure (state_conversions.hpp:9-24).
__device__ __forceinline__ double pressure_of(const GasParams& g, const double U[5]) {
    const double rho = U[0];
    const double inv_rho = 1.0 / rho;
    const double q2 = (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) * (inv_rho * inv_rho);
    const double e = (U[4] * inv_rho) - 0.5 * q2;
    return (g.gamma - 1.0) * rho * e;
}

// ViscousFlux::viscosity, Sutherland (fluxes/viscous.hpp:68-74).
__device__ __forceinline__ double sutherland(double T) {
    const double c = kSuthMu * (kSuthTRef + kSuthS);
    const double ratio = T / kSuthTRef;
    return c * ratio * sqrt(ratio) / (T + kSuthS);
}

// ---------------------------------------------------------------- HLLC
// HllcFlux::star_flux (fluxes/hllc.hpp:231-274).
__device__ __forceinline__ void hllc_star(const double UK[5], const double FK[5], double rhoK, double pK, double ux,
                                          double uy, double uz, double unk, double ak, double SK, double SM,
                                          double nx, double ny, double nz, double area, double F[5]) {
    const double den = SK - SM;
    if (fabs(den) < 1.0e-6 * (ak + fabs(SK))) {
        for (int v = 0; v < 5; ++v) F[v] = FK[v] * area;
        return;
    }
    const double inv_den = 1.0 / den;
    const double d_wave = SK - unk;
    const double q = d_wave * inv_den;
    const double d = SM - unk;
    const double p_term = pK / (rhoK * d_wave);
    const double e_star = UK[4] + rhoK * d * (SM + p_term);
    const double Ust[5] = {q * rhoK, q * rhoK * (ux + d * nx), q * rhoK * (uy + d * ny), q * rhoK * (uz + d * nz),
                           q * e_star};
    for (int v = 0; v < 5; ++v) F[v] = (FK[v] + SK * (Ust[v] - UK[v])) * area;
}

// HllcFlux::face_flux: HLLC with Roe/Einfeldt outer waves (fluxes/hllc.hpp:21-122).
__device__ __forceinline__ void hllc_flux(const GasParams& g, const double UL[5], const double UR[5], double nx,
                                          double ny, double nz, double area, double F[5], double& smax) {
    const double rhoL = UL[0], rhoR = UR[0];
    const double inv_rhoL = 1.0 / rhoL, inv_rhoR = 1.0 / rhoR;
    const double pL = pressure_of(g, UL), pR = pressure_of(g, UR);
    const double uLx = UL[1] * inv_rhoL, uLy = UL[2] * inv_rhoL, uLz = UL[3] * inv_rhoL;
    const double uRx = UR[1] * inv_rhoR, uRy = UR[2] * inv_rhoR, uRz = UR[3] * inv_rhoR;
    const double unL = uLx * nx + uLy * ny + uLz * nz;
    const double unR = uRx * nx + uRy * ny + uRz * nz;
    const double aL = sqrt(g.gamma * pL / rhoL);
    const double aR = sqrt(g.gamma * pR / rhoR);
    const double rl = sqrt(rhoL), rr = sqrt(rhoR);
    const double w = 1.0 / (rl + rr);
    const double roe_ux = (rl * uLx + rr * uRx) * w;
    const double roe_uy = (rl * uLy + rr * uRy) * w;
    const double roe_uz = (rl * uLz + rr * uRz) * w;
    const double HL = (UL[4] + pL) * inv_rhoL;
    const double HR = (UR[4] + pR) * inv_rhoR;
    const double roe_h = (rl * HL + rr * HR) * w;
    const double q2 = roe_ux * roe_ux + roe_uy * roe_uy + roe_uz * roe_uz;
    const double a2 = (g.gamma - 1.0) * (roe_h - 0.5 * q2);
    const double roe_a = sqrt(a2 > 0.0 ? a2 : 0.0);
    const double roe_un = roe_ux * nx + roe_uy * ny + roe_uz * nz;
    const double SL = fmin(unL - aL, roe_un - roe_a);
    const double SR = fmax(unR + aR, roe_un + roe_a);
    smax = fmax(fabs(SL), fabs(SR));
    const double dL = SL - unL, dR = SR - unR;
    const double denom = rhoL * dL - rhoR * dR;
    const double SM = (fabs(denom) > 1e-14) ? (pR - pL + rhoL * unL * dL - rhoR * unR * dR) / denom : 0.5 * (unL + unR);
    if (SM >= 0.0) {
        const double FL[5] = {rhoL * unL, rhoL * uLx * unL + pL * nx, rhoL * uLy * unL + pL * ny,
                              rhoL * uLz * unL + pL * nz, (UL[4] + pL) * unL};
        if (SL >= 0.0) {
            for (int v = 0; v < 5; ++v) F[v] = FL[v] * area;
        } else {
            hllc_star(UL, FL, rhoL, pL, uLx, uLy, uLz, unL, aL, SL, SM, nx, ny, nz, area, F);
        }
    } else {
        const double FR[5] = {rhoR * unR, rhoR * uRx * unR + pR * nx, rhoR * uRy * unR + pR * ny,
                              rhoR * uRz * unR + pR * nz, (UR[4] + pR) * unR};
        if (SR <= 0.0) {
            for (int v = 0; v < 5; ++v) F[v] = FR[v] * area;
        } else {
            hllc_star(UR, FR, rhoR, pR, uRx, uRy, uRz, unR, aR, SR, SM, nx, ny, nz, area, F);
        }
    }
}

// Only the wave-speed bound of hllc_flux (used by the Jacobian, which needs
// s_max of a full face_flux call, fluxes/hllc.hpp:144-147).
__device__ __forceinline__ double hllc_smax(const GasParams& g, const double UL[5], const double UR[5], double nx,
                                            double ny, double nz) {
    const double rhoL = UL[0], rhoR = UR[0];
    const double inv_rhoL = 1.0 / rhoL, inv_rhoR = 1.0 / rhoR;
    const double pL = pressure_of(g, UL), pR = pressure_of(g, UR);
    const double uLx = UL[1] * inv_rhoL, uLy = UL[2] * inv_rhoL, uLz = UL[3] * inv_rhoL;
    const double uRx = UR[1] * inv_rhoR, uRy = UR[2] * inv_rhoR, uRz = UR[3] * inv_rhoR;
    const double unL = uLx * nx + uLy * ny + uLz * nz;
    const double unR = uRx * nx + uRy * ny + uRz * nz;
    const double aL = sqrt(g.gamma * pL / rhoL);
    const double aR = sqrt(g.gamma * pR / rhoR);
    const double rl = sqrt(rhoL), rr = sqrt(rhoR);
    const double w = 1.0 / (rl + rr);
    const double roe_ux = (rl * uLx + rr * uRx) * w;
    const double roe_uy = (rl * uLy + rr * uRy) * w;
    const double roe_uz = (rl * uLz + rr * uRz) * w;
    const double HL = (UL[4] + pL) * inv_rhoL;
    const double HR = (UR[4] + pR) * inv_rhoR;
    const double roe_h = (rl * HL + rr * HR) * w;
    const double q2 = roe_ux * roe_ux + roe_uy * roe_uy + roe_uz * roe_uz;
    const double a2 = (g.gamma - 1.0) * (roe_h - 0.5 * q2);
    const double roe_a = sqrt(a2 > 0.0 ? a2 : 0.0);
    const double roe_un = roe_ux * nx + roe_uy * ny + roe_uz * nz;
    const double SL = fmin(unL - aL, roe_un - roe_a);
    const double SR = fmax(unR + aR, roe_un + roe_a);
    return fmax(fabs(SL), fabs(SR));
}

// Exact Jacobian of the normal Euler flux, row-major 5x5, scaled by s
// (HllcFlux::analytical_physical_jacobian, fluxes/hllc.hpp:172-229).
__device__ __forceinline__ void euler_jacobian(const GasParams& g, const double U[5], double nx, double ny, double nz,
                                               double J[25]) {
    const double rho = U[0];
    const double inv_rho = 1.0 / rho;
    const double u = U[1] * inv_rho, v = U[2] * inv_rho, w = U[3] * inv_rho, E = U[4] * inv_rho;
    const double p = pressure_of(g, U);
    const double gamma = g.gamma, phi = gamma - 1.0;
    const double un = u * nx + v * ny + w * nz;
    const double q2 = u * u + v * v + w * w;
    const double H = E + p * inv_rho;
    const double hpq = 0.5 * phi * q2;
    J[0] = 0.0;
    J[1] = nx;
    J[2] = ny;
    J[3] = nz;
    J[4] = 0.0;
    J[5] = hpq * nx - u * un;
    J[6] = un + nx * (1.0 - phi) * u;
    J[7] = u * ny - phi * nx * v;
    J[8] = u * nz - phi * nx * w;
    J[9] = phi * nx;
    J[10] = hpq * ny - v * un;
    J[11] = v * nx - phi * ny * u;
    J[12] = un + ny * (1.0 - phi) * v;
    J[13] = v * nz - phi * ny * w;
    J[14] = phi * ny;
    J[15] = hpq * nz - w * un;
    J[16] = w * nx - phi * nz * u;
    J[17] = w * ny - phi * nz * v;
    J[18] = un + nz * (1.0 - phi) * w;
    J[19] = phi * nz;
    J[20] = un * (hpq - H);
    J[21] = H * nx - phi * u * un;
    J[22] = H * ny - phi * v * un;
    J[23] = H * nz - phi * w * un;
    J[24] = gamma * un;
}

// ------------------------------------------------------------- viscous
struct ViscGeom {
    double inv_d, dx, dy, dz;
};

// ViscousFlux::face_flux (fluxes/viscous.hpp:90-175) from cell-centre
// primitives qL/qR and the 12 gradient components [du, dv, dw, dT] of both
// sides.  Fv[0] stays 0; returns lam_visc.
__device__ __forceinline__ double viscous_flux(const GasParams& g, const ViscGeom& geo, const double qL[5],
                                               const double qR[5], const double gL[12], const double gR[12],
                                               double mutL, double mutR, double nx, double ny, double nz, double area,
                                               double Fv[5]) {
    const double p_f = 0.5 * (qL[0] + qR[0]);
    const double u_f = 0.5 * (qL[1] + qR[1]);
    const double v_f = 0.5 * (qL[2] + qR[2]);
    const double w_f = 0.5 * (qL[3] + qR[3]);
    const double T_f = 0.5 * (qL[4] + qR[4]);
    const double mu_lam = sutherland(T_f);
    const double mu_t_f = 0.5 * (mutL + mutR);
    const double mu_eff = mu_lam + mu_t_f;
    const double k_lam = (mu_lam * g.cp) / g.prandtl;
    const double k_eff = k_lam + (mu_t_f * g.cp) / g.prandtl_turb;
    const double inv_d = geo.inv_d;
    const double xi_x = geo.dx * inv_d, xi_y = geo.dy * inv_d, xi_z = geo.dz * inv_d;
    const double ncx = nx - xi_x, ncy = ny - xi_y, ncz = nz - xi_z;
    const double du_dx = 0.5 * (gL[0] + gR[0]), du_dy = 0.5 * (gL[1] + gR[1]), du_dz = 0.5 * (gL[2] + gR[2]);
    const double dv_dx = 0.5 * (gL[3] + gR[3]), dv_dy = 0.5 * (gL[4] + gR[4]), dv_dz = 0.5 * (gL[5] + gR[5]);
    const double dw_dx = 0.5 * (gL[6] + gR[6]), dw_dy = 0.5 * (gL[7] + gR[7]), dw_dz = 0.5 * (gL[8] + gR[8]);
    const double dT_dx = 0.5 * (gL[9] + gR[9]), dT_dy = 0.5 * (gL[10] + gR[10]), dT_dz = 0.5 * (gL[11] + gR[11]);
    const double div_v = du_dx + dv_dy + dw_dz;
    const double ttd = (2.0 / 3.0) * div_v;
    const double du_dn = (qR[1] - qL[1]) * inv_d + (du_dx * ncx + du_dy * ncy + du_dz * ncz);
    const double dv_dn = (qR[2] - qL[2]) * inv_d + (dv_dx * ncx + dv_dy * ncy + dv_dz * ncz);
    const double dw_dn = (qR[3] - qL[3]) * inv_d + (dw_dx * ncx + dw_dy * ncy + dw_dz * ncz);
    const double dT_dn = (qR[4] - qL[4]) * inv_d + (dT_dx * ncx + dT_dy * ncy + dT_dz * ncz);
    const double tnx = mu_eff * (du_dn + (du_dx * nx + dv_dx * ny + dw_dx * nz) - ttd * nx);
    const double tny = mu_eff * (dv_dn + (du_dy * nx + dv_dy * ny + dw_dy * nz) - ttd * ny);
    const double tnz = mu_eff * (dw_dn + (du_dz * nx + dv_dz * ny + dw_dz * nz) - ttd * nz);
    const double qn = -k_eff * dT_dn;
    const double rho_f = p_f / (g.R * T_f);
    const double nu_eff = mu_eff / rho_f;
    Fv[0] = 0.0;
    Fv[1] = -tnx * area;
    Fv[2] = -tny * area;
    Fv[3] = -tnz * area;
    Fv[4] = (-(u_f * tnx + v_f * tny + w_f * tnz) + qn) * area;
    return (4.0 / 3.0) * nu_eff * inv_d * area;
}

// ViscousFlux::face_flux_jacobian, thin-layer dFv/dUL (dFv/dUR = -dFv/dUL)
// (fluxes/viscous.hpp:280-360).  Accumulates into J with factor s.
//
// FULL adds the normal-stress term of the thin-layer operator,
// d tau / d u = mu/d (I + n n^T / 3), which the reference drops (so the
// normal momentum sees 3/4 of its viscous stiffness).  wv and wt scale the
// velocity and temperature derivatives: 2 on a no-slip wall face whose
// ghost mirrors the velocity (u_g = 2 u_w - u) or the temperature
// (isothermal, T_g = 2 T_w - T), 1 elsewhere.
template <bool FULL>
__device__ __forceinline__ void viscous_jacobian_add(const GasParams& g, double inv_d, const double qL[5],
                                                     const double qR[5], double mutL, double mutR, double area,
                                                     double s, double J[25], double nx = 0.0, double ny = 0.0,
                                                     double nz = 0.0, double wv = 1.0, double wt = 1.0) {
    const double p_f = 0.5 * (qL[0] + qR[0]);
    const double u_f = 0.5 * (qL[1] + qR[1]);
    const double v_f = 0.5 * (qL[2] + qR[2]);
    const double w_f = 0.5 * (qL[3] + qR[3]);
    const double T_f = 0.5 * (qL[4] + qR[4]);
    const double rho_f = p_f / (g.R * T_f);
    const double inv_rho = 1.0 / rho_f;
    const double cv = g.cv;
    const double inv_rho_cv = 1.0 / (rho_f * cv);
    const double mu_lam = sutherland(T_f);
    const double mu_t_f = 0.5 * (mutL + mutR);
    const double mu_eff = mu_lam + mu_t_f;
    const double k_lam = (mu_lam * g.cp) / g.prandtl;
    const double k_eff = k_lam + (mu_t_f * g.cp) / g.prandtl_turb;
    const double C_mu = mu_eff * inv_d * area;
    const double C_lam = k_eff * inv_d * area;
    const double V2 = u_f * u_f + v_f * v_f + w_f * w_f;
    if (!FULL) {
        J[5] += s * (-C_mu * u_f * inv_rho);
        J[6] += s * (C_mu * inv_rho);
        J[10] += s * (-C_mu * v_f * inv_rho);
        J[12] += s * (C_mu * inv_rho);
        J[15] += s * (-C_mu * w_f * inv_rho);
        J[18] += s * (C_mu * inv_rho);
        J[20] += s * (C_lam * (0.5 * V2 - cv * T_f) * inv_rho_cv - C_mu * V2 * inv_rho);
        J[21] += s * (-C_lam * u_f * inv_rho_cv + C_mu * u_f * inv_rho);
        J[22] += s * (-C_lam * v_f * inv_rho_cv + C_mu * v_f * inv_rho);
        J[23] += s * (-C_lam * w_f * inv_rho_cv + C_mu * w_f * inv_rho);
        J[24] += s * (C_lam * inv_rho_cv);
    } else {
        const double n[3] = {nx, ny, nz}, u[3] = {u_f, v_f, w_f};
        const double un3 = (nx * u_f + ny * v_f + nz * w_f) * (1.0 / 3.0);
        const double cm = wv * C_mu, cl = wt * C_lam;
        double Mu[3];  // (I + n n^T / 3) u
#pragma unroll
        for (int a = 0; a < 3; ++a) Mu[a] = u[a] + n[a] * un3;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            J[(1 + a) * 5] += s * (-cm * Mu[a] * inv_rho);
#pragma unroll
            for (int b = 0; b < 3; ++b)
                J[(1 + a) * 5 + 1 + b] += s * (cm * ((a == b ? 1.0 : 0.0) + n[a] * n[b] * (1.0 / 3.0)) * inv_rho);
        }
        const double uMu = u_f * Mu[0] + v_f * Mu[1] + w_f * Mu[2];
        J[20] += s * (cl * (0.5 * V2 - cv * T_f) * inv_rho_cv - cm * uMu * inv_rho);
#pragma unroll
        for (int b = 0; b < 3; ++b) J[21 + b] += s * (-cl * u[b] * inv_rho_cv + cm * Mu[b] * inv_rho);
        J[24] += s * (cl * inv_rho_cv);
    }
}

// ------------------------------------------------------------- limiters
// MultidimSlopeLimiter::phi (numerics/limiter/slope_limiters.hpp:21-79).
template <int LIM>
__device__ __forceinline__ double limiter_phi(double dnb, double df, double eps2) {
    if (df == 0.0) return 1.0;
    if (LIM == 2) {  // Barth-Jespersen
        const double r = dnb / df;
        return fmin(fmax(r, 0.0), 1.0);
    }
    const double prod = dnb * df;
    if (prod <= 0.0) return 0.0;
    if (LIM == 3) {  // Van Albada
        const double num = dnb * dnb + prod;
        const double den = dnb * dnb + df * df + eps2;
        return (den > 0.0) ? (num / den) : 1.0;
    }
    // Venkatakrishnan
    const double a2 = dnb * dnb + eps2;
    const double num = a2 + 2.0 * prod;
    const double den = a2 + 2.0 * df * df + prod;
    return num / den;
}

// ------------------------------------------------------- boundary rules
// compute_riemann_farfield_state (bc/physical/farfield.hpp:39-100).
__device__ __forceinline__ bool farfield_state(const BcPatch& P, const GasParams& g, double p_in, double T_in,
                                               double vx_in, double vy_in, double vz_in, double nx, double ny,
                                               double nz, double qb[5]) {
    const double gamma = g.gamma, R = g.R;
    const double gm1 = gamma - 1.0;
    const double inv_gm1 = 1.0 / gm1;
    const double un_in = vx_in * nx + vy_in * ny + vz_in * nz;
    const double un_inf = P.far_u * nx + P.far_v * ny + P.far_w * nz;
    const double a_in = sqrt(gamma * R * fmax(T_in, 1.0e-6));
    const double a_inf = sqrt(gamma * R * fmax(P.far_T, 1.0e-6));
    const double mn_in = un_in / a_in;
    if (mn_in >= 1.0) {
        qb[0] = p_in;
        qb[1] = vx_in;
        qb[2] = vy_in;
        qb[3] = vz_in;
        qb[4] = T_in;
        return true;
    }
    if (mn_in <= -1.0) {
        qb[0] = P.far_p;
        qb[1] = P.far_u;
        qb[2] = P.far_v;
        qb[3] = P.far_w;
        qb[4] = P.far_T;
        return false;
    }
    const double R_out = un_in + 2.0 * a_in * inv_gm1;
    const double R_in = un_inf - 2.0 * a_inf * inv_gm1;
    const double un_b = 0.5 * (R_out + R_in);
    double a_b = 0.25 * gm1 * (R_out - R_in);
    if (a_b <= 0.0) a_b = a_inf;
    double entropy_s;
    if (un_b >= 0.0) {
        qb[1] = vx_in + (un_b - un_in) * nx;
        qb[2] = vy_in + (un_b - un_in) * ny;
        qb[3] = vz_in + (un_b - un_in) * nz;
        const double rho_in = p_in / (R * fmax(T_in, 1.0e-6));
        entropy_s = p_in / pow(fmax(rho_in, 1.0e-12), gamma);
    } else {
        qb[1] = P.far_u + (un_b - un_inf) * nx;
        qb[2] = P.far_v + (un_b - un_inf) * ny;
        qb[3] = P.far_w + (un_b - un_inf) * nz;
        const double rho_inf = P.far_p / (R * fmax(P.far_T, 1.0e-6));
        entropy_s = P.far_p / pow(fmax(rho_inf, 1.0e-12), gamma);
    }
    const double rho_b = pow((a_b * a_b) / (gamma * fmax(entropy_s, 1.0e-12)), inv_gm1);
    qb[0] = (rho_b * a_b * a_b) / gamma;
    qb[4] = (a_b * a_b) / (gamma * R);
    return false;
}

// Ghost primitive state of one boundary face: the update_ghost_cells kernels
// of the nine BC classes (bc/physical/*.hpp, numerics/boundary/boundary_values.hpp).
// rcfn = (x_f - x_c).n of the owner.
__device__ __forceinline__ void ghost_values(const BcPatch& P, const GasParams& g, const double qi[5], double nx,
                                             double ny, double nz, double rcfn, double qg[5]) {
    switch (P.kind) {
        case 0: {  // SUPERSONIC_INLET
            for (int v = 0; v < 5; ++v) qg[v] = 2.0 * P.qfix[v] - qi[v];
            qg[0] = fmax(qg[0], 1.0);
            qg[4] = fmax(qg[4], 1.0);
            break;
        }
        case 1:  // SUPERSONIC_OUTLET
            for (int v = 0; v < 5; ++v) qg[v] = qi[v];
            break;
        case 4:    // SLIP_WALL
        case 7: {  // SYMMETRY
            const double vn2 = 2.0 * (qi[1] * nx + qi[2] * ny + qi[3] * nz);
            qg[1] = qi[1] - vn2 * nx;
            qg[2] = qi[2] - vn2 * ny;
            qg[3] = qi[3] - vn2 * nz;
            qg[0] = qi[0];
            qg[4] = qi[4];
            break;
        }
        case 8: {  // FARFIELD
            double qb[5];
            const bool sup_out = farfield_state(P, g, qi[0], qi[4], qi[1], qi[2], qi[3], nx, ny, nz, qb);
            if (sup_out) {
                for (int v = 0; v < 5; ++v) qg[v] = qi[v];
            } else {
                for (int v = 0; v < 5; ++v) qg[v] = 2.0 * qb[v] - qi[v];
                qg[0] = fmax(qg[0], 1.0);
                qg[4] = fmax(qg[4], 1.0);
            }
            break;
        }
        case 5: {  // NO_SLIP_WALL (isothermal)
            qg[0] = qi[0];
            qg[1] = 2.0 * P.qfix[1] - qi[1];
            qg[2] = 2.0 * P.qfix[2] - qi[2];
            qg[3] = 2.0 * P.qfix[3] - qi[3];
            qg[4] = fmax(2.0 * P.qfix[4] - qi[4], 1.0);
            break;
        }
        case 6: {  // NO_SLIP_WALL_HEAT_FLUX
            qg[0] = qi[0];
            qg[1] = 2.0 * P.qfix[1] - qi[1];
            qg[2] = 2.0 * P.qfix[2] - qi[2];
            qg[3] = 2.0 * P.qfix[3] - qi[3];
            const double rcfn_inv = 1.0 / fmax(rcfn, 1.0e-14);
            const double r = 1.0 / rcfn_inv;
            qg[4] = fmax(qi[4] + 2.0 * P.tmp_grad * r, 1.0);
            break;
        }
        case 2: {  // SUBSONIC_INLET
            qg[0] = qi[0];
            qg[1] = 2.0 * P.qfix[1] - qi[1];
            qg[2] = 2.0 * P.qfix[2] - qi[2];
            qg[3] = 2.0 * P.qfix[3] - qi[3];
            qg[4] = fmax(2.0 * P.qfix[4] - qi[4], 1.0);
            break;
        }
        case 3: {  // SUBSONIC_OUTLET
            qg[0] = fmax(2.0 * P.p_out - qi[0], 1.0);
            for (int v = 1; v < 5; ++v) qg[v] = qi[v];
            break;
        }
        default:
            for (int v = 0; v < 5; ++v) qg[v] = qi[v];
            break;
    }
}

// numerics/boundary/boundary_gradients.hpp:15-160.
__device__ __forceinline__ void grad_dirichlet(const double gi[3], double qin, double qfix, double nx, double ny,
                                               double nz, double rcfn_inv, double gg[3]) {
    const double ddn = (qfix - qin) * rcfn_inv;
    const double gdn = gi[0] * nx + gi[1] * ny + gi[2] * nz;
    const double f = 2.0 * (ddn - gdn);
    gg[0] = gi[0] + f * nx;
    gg[1] = gi[1] + f * ny;
    gg[2] = gi[2] + f * nz;
}
__device__ __forceinline__ void grad_neumann(const double gi[3], double fixed, double nx, double ny, double nz,
                                             double gg[3]) {
    const double gdn = gi[0] * nx + gi[1] * ny + gi[2] * nz;
    const double f = 2.0 * (fixed - gdn);
    gg[0] = gi[0] + f * nx;
    gg[1] = gi[1] + f * ny;
    gg[2] = gi[2] + f * nz;
}
__device__ __forceinline__ void grad_slip(const double gi[3], double qin, double qgh, double nx, double ny, double nz,
                                          double rcfn_inv, double gg[3]) {
    const double gdn = gi[0] * nx + gi[1] * ny + gi[2] * nz;
    const double ddn = 0.5 * (qgh - qin) * rcfn_inv;
    const double f = 2.0 * (ddn - gdn);
    gg[0] = gi[0] + f * nx;
    gg[1] = gi[1] + f * ny;
    gg[2] = gi[2] + f * nz;
}

// Ghost gradients of the 5 mean-flow primitives for one boundary face: the
// update_ghost_cells_grad kernels of the nine BC classes.  gi[v][3] interior
// gradients, qi/qgh interior and ghost primitives.
__device__ __forceinline__ void ghost_gradients(const BcPatch& P, const GasParams& g, const double gi[5][3],
                                                const double qi[5], const double qgh[5], double nx, double ny,
                                                double nz, double rcfn_inv, double gg[5][3]) {
    switch (P.kind) {
        case 0:  // SUPERSONIC_INLET: Dirichlet on all
            for (int v = 0; v < 5; ++v) grad_dirichlet(gi[v], qi[v], P.qfix[v], nx, ny, nz, rcfn_inv, gg[v]);
            break;
        case 1:  // SUPERSONIC_OUTLET: extrapolate
            for (int v = 0; v < 5; ++v)
                for (int d = 0; d < 3; ++d) gg[v][d] = gi[v][d];
            break;
        case 4:
        case 7:  // SLIP_WALL / SYMMETRY
            grad_neumann(gi[0], 0.0, nx, ny, nz, gg[0]);
            for (int v = 1; v < 4; ++v) grad_slip(gi[v], qi[v], qgh[v], nx, ny, nz, rcfn_inv, gg[v]);
            grad_neumann(gi[4], 0.0, nx, ny, nz, gg[4]);
            break;
        case 8: {  // FARFIELD
            double qb[5];
            const bool sup_out = farfield_state(P, g, qi[0], qi[4], qi[1], qi[2], qi[3], nx, ny, nz, qb);
            if (sup_out) {
                for (int v = 0; v < 5; ++v)
                    for (int d = 0; d < 3; ++d) gg[v][d] = gi[v][d];
            } else {
                for (int v = 0; v < 5; ++v) grad_dirichlet(gi[v], qi[v], qb[v], nx, ny, nz, rcfn_inv, gg[v]);
            }
            break;
        }
        case 5:  // NO_SLIP_WALL
        case 2:  // SUBSONIC_INLET
            for (int d = 0; d < 3; ++d) gg[0][d] = gi[0][d];
            for (int v = 1; v < 5; ++v) grad_dirichlet(gi[v], qi[v], P.qfix[v], nx, ny, nz, rcfn_inv, gg[v]);
            break;
        case 6:  // NO_SLIP_WALL_HEAT_FLUX
            for (int d = 0; d < 3; ++d) gg[0][d] = gi[0][d];
            for (int v = 1; v < 4; ++v) grad_dirichlet(gi[v], qi[v], P.qfix[v], nx, ny, nz, rcfn_inv, gg[v]);
            grad_neumann(gi[4], P.tmp_grad, nx, ny, nz, gg[4]);
            break;
        case 3:  // SUBSONIC_OUTLET
            grad_dirichlet(gi[0], qi[0], P.p_out, nx, ny, nz, rcfn_inv, gg[0]);
            for (int v = 1; v < 5; ++v)
                for (int d = 0; d < 3; ++d) gg[v][d] = gi[v][d];
            break;
        default:
            for (int v = 0; v < 5; ++v)
                for (int d = 0; d < 3; ++d) gg[v][d] = gi[v][d];
            break;
    }
}

}  // namespace cfdg
