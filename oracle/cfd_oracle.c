/*
 * CPU restatement of the implicit compressible finite-volume hot path of
 * maksim-movsisyan/Distributed-cfd-solver (single partition, np = 1).
 * TEST INFRASTRUCTURE ONLY (see cfd_oracle.h).  Each function names the
 * reference routine whose algorithm it restates.  Face loops scatter into
 * cells sequentially in face order, as the reference does, so the results
 * are the reference's up to floating-point contraction.
 */
#include "cfd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_PI 3.14159265358979323846
#define SUTH_MU 1.716e-5
#define SUTH_TREF 273.15
#define SUTH_S 110.4

typedef struct {
    int kind;
    int sa_kind; /* SpalartAllmaras::zone_kind: 0 wall, 1 inflow, 2 outflow, 3 symmetry */
    double qfix[5], p_out, tmp_grad, far_p, far_T, far_u, far_v, far_w;
} bcp_t;

/* Spalart & Allmaras (1994) constants (spalart_allmaras.hpp:85-93). */
#define SA_CB1 0.1355
#define SA_CB2 0.622
#define SA_SIGMA (2.0 / 3.0)
#define SA_KAPPA 0.41
#define SA_CW2 0.3
#define SA_CW3 2.0
#define SA_CV1 7.1
#define SA_CW1 (SA_CB1 / (SA_KAPPA * SA_KAPPA) + (1.0 + SA_CB2) / SA_SIGMA)
#define SA_SBAR_FLOOR 1.0e-10
#define SA_MIN_WALL_DIST 1.0e-10

struct oracle_solver {
    cfdg_mesh_host m;
    cfdg_config cfg;
    double gamma, R, cv, cp;
    int n, nf, ni, nb, nt, nv;
    int muscl, visc, need_grad;
    bcp_t* bcp;
    int n_patch;
    int32_t *c2f_off, *c2f, *c2c_off, *c2c, *g_off, *g_col;
    double *g_wx, *g_wy, *g_wz;
    double *fdx, *fdy, *fdz, *finv_d;
    int32_t *rp, *cols, *diag;
    int64_t nnzb;
    double *U, *q, *grad, *phi, *res, *lam, *alpha, *vals;
    int phi_frozen; /* limiter values kept from the last evaluation (cfdg_solver_freeze_limiter) */
    /* Spalart-Allmaras */
    int sa;
    double nu_inf, rhonu_inf;
    double *dist, *nu, *rho, *mut, *gnu, *mdot, *rhonu_g;
};

static void* xcalloc(size_t n, size_t s) { return calloc(n ? n : 1, s); }

/* ------------------------------------------------------------ connectivity */
/* build_cell_faces_conn / build_cell_cells_face_conn / build_cell_cells_node_conn
 * (src/mesh/aux_connectivity.cpp:11-187, 290-445). */
static int cmp_i32(const void* a, const void* b) {
    const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

int64_t oracle_connectivity(const cfdg_mesh_host* m, int kind, int32_t* off, int32_t* val) {
    const int n = m->n_cells, nf = m->n_faces;
    int32_t* cnt = (int32_t*)xcalloc((size_t)n + 1, sizeof(int32_t));
    int64_t total = 0;
    if (kind == 0 || kind == 1) {
        for (int f = 0; f < nf; ++f) {
            const int o = m->face_owner[f], g = m->face_neigh[f];
            if (kind == 1 && g < 0) continue;
            cnt[o + 1]++;
            if (g >= 0) cnt[g + 1]++;
        }
        for (int c = 0; c < n; ++c) cnt[c + 1] += cnt[c];
        total = cnt[n];
        if (off) memcpy(off, cnt, sizeof(int32_t) * ((size_t)n + 1));
        if (val) {
            int32_t* cur = (int32_t*)xcalloc((size_t)n, sizeof(int32_t));
            for (int c = 0; c < n; ++c) cur[c] = cnt[c];
            for (int f = 0; f < nf; ++f) {
                const int o = m->face_owner[f], g = m->face_neigh[f];
                if (kind == 1 && g < 0) continue;
                val[cur[o]++] = (kind == 0) ? f : g;
                if (g >= 0) val[cur[g]++] = (kind == 0) ? f : o;
            }
            if (kind == 1)
                for (int c = 0; c < n; ++c) qsort(val + cnt[c], (size_t)(cnt[c + 1] - cnt[c]), sizeof(int32_t), cmp_i32);
            free(cur);
        }
        free(cnt);
        return total;
    }
    /* node stencil */
    const int nn = m->n_nodes;
    int32_t* n2c_off = (int32_t*)xcalloc((size_t)nn + 1, sizeof(int32_t));
    const int32_t* co = m->cell_nodes_offsets;
    for (int c = 0; c < n; ++c)
        for (int k = co[c]; k < co[c + 1]; ++k) n2c_off[m->cell_nodes[k] + 1]++;
    for (int i = 0; i < nn; ++i) n2c_off[i + 1] += n2c_off[i];
    int32_t* n2c = (int32_t*)xcalloc((size_t)n2c_off[nn], sizeof(int32_t));
    int32_t* cur = (int32_t*)xcalloc((size_t)nn, sizeof(int32_t));
    for (int i = 0; i < nn; ++i) cur[i] = n2c_off[i];
    for (int c = 0; c < n; ++c)
        for (int k = co[c]; k < co[c + 1]; ++k) n2c[cur[m->cell_nodes[k]]++] = c;
    int32_t* stamp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
    for (int c = 0; c < n; ++c) stamp[c] = -1;
    int32_t* buf = (int32_t*)malloc(sizeof(int32_t) * 1024);
    int64_t w = 0;
    if (off) off[0] = 0;
    for (int c = 0; c < n; ++c) {
        int nb = 0;
        for (int k = co[c]; k < co[c + 1]; ++k) {
            const int node = m->cell_nodes[k];
            for (int j = n2c_off[node]; j < n2c_off[node + 1]; ++j) {
                const int o = n2c[j];
                if (o == c || stamp[o] == c) continue;
                stamp[o] = c;
                buf[nb++] = o;
            }
        }
        qsort(buf, (size_t)nb, sizeof(int32_t), cmp_i32);
        if (val) memcpy(val + w, buf, sizeof(int32_t) * (size_t)nb);
        w += nb;
        if (off) off[c + 1] = (int32_t)w;
    }
    free(buf);
    free(stamp);
    free(cur);
    free(n2c);
    free(n2c_off);
    free(cnt);
    return w;
}

/* ------------------------------------------------------------------ EOS */
/* eos::primitives_pT_to_conserved / conserved_to_primitives_pT / pressure
 * (include/cfd/solver/compressible/eos/state_conversions.hpp:9-129). */
static void prim2cons(const oracle_solver* s, const double* q, double* U) {
    const double rho = q[0] / (s->R * q[4]);
    const double e = s->cv * q[4];
    const double ke = 0.5 * rho * (q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    U[0] = rho;
    U[1] = rho * q[1];
    U[2] = rho * q[2];
    U[3] = rho * q[3];
    U[4] = rho * e + ke;
}

static void cons2prim(const oracle_solver* s, const double* U, double* q) {
    const double rho = U[0], ir = 1.0 / rho;
    const double u = U[1] * ir, v = U[2] * ir, w = U[3] * ir;
    const double e = U[4] * ir - 0.5 * (u * u + v * v + w * w);
    q[0] = (s->gamma - 1.0) * rho * e;
    q[1] = u;
    q[2] = v;
    q[3] = w;
    q[4] = e / s->cv;
}

static double pressure(const oracle_solver* s, const double* U) {
    const double rho = U[0], ir = 1.0 / rho;
    const double q2 = (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) * (ir * ir);
    return (s->gamma - 1.0) * rho * (U[4] * ir - 0.5 * q2);
}

static double sutherland(double T) {
    const double c = SUTH_MU * (SUTH_TREF + SUTH_S);
    const double r = T / SUTH_TREF;
    return c * r * sqrt(r) / (T + SUTH_S);
}

/* ------------------------------------------------------------------ HLLC */
/* HllcFlux::face_flux + star_flux (fluxes/hllc.hpp:21-122, 231-274). */
static void star(const double* UK, const double* FK, double rhoK, double pK, double ux, double uy, double uz,
                 double unk, double ak, double SK, double SM, double nx, double ny, double nz, double A, double* F) {
    const double den = SK - SM;
    if (fabs(den) < 1.0e-6 * (ak + fabs(SK))) {
        for (int v = 0; v < 5; ++v) F[v] = FK[v] * A;
        return;
    }
    const double q = (SK - unk) / den;
    const double d = SM - unk;
    const double e_star = UK[4] + rhoK * d * (SM + pK / (rhoK * (SK - unk)));
    const double Ust[5] = {q * rhoK, q * rhoK * (ux + d * nx), q * rhoK * (uy + d * ny), q * rhoK * (uz + d * nz),
                           q * e_star};
    for (int v = 0; v < 5; ++v) F[v] = (FK[v] + SK * (Ust[v] - UK[v])) * A;
}

static void hllc(const oracle_solver* s, const double* UL, const double* UR, double nx, double ny, double nz,
                 double A, double* F, double* smax) {
    const double g = s->gamma;
    const double rL = UL[0], rR = UR[0];
    const double pL = pressure(s, UL), pR = pressure(s, UR);
    const double uLx = UL[1] / rL, uLy = UL[2] / rL, uLz = UL[3] / rL;
    const double uRx = UR[1] / rR, uRy = UR[2] / rR, uRz = UR[3] / rR;
    const double unL = uLx * nx + uLy * ny + uLz * nz, unR = uRx * nx + uRy * ny + uRz * nz;
    const double aL = sqrt(g * pL / rL), aR = sqrt(g * pR / rR);
    const double sl = sqrt(rL), sr = sqrt(rR), w = 1.0 / (sl + sr);
    const double ux = (sl * uLx + sr * uRx) * w, uy = (sl * uLy + sr * uRy) * w, uz = (sl * uLz + sr * uRz) * w;
    const double H = (sl * (UL[4] + pL) / rL + sr * (UR[4] + pR) / rR) * w;
    const double a2 = (g - 1.0) * (H - 0.5 * (ux * ux + uy * uy + uz * uz));
    const double a = sqrt(a2 > 0.0 ? a2 : 0.0);
    const double un = ux * nx + uy * ny + uz * nz;
    const double SL = fmin(unL - aL, un - a), SR = fmax(unR + aR, un + a);
    *smax = fmax(fabs(SL), fabs(SR));
    const double dL = SL - unL, dR = SR - unR, den = rL * dL - rR * dR;
    const double SM = (fabs(den) > 1e-14) ? (pR - pL + rL * unL * dL - rR * unR * dR) / den : 0.5 * (unL + unR);
    if (SM >= 0.0) {
        const double FL[5] = {rL * unL, rL * uLx * unL + pL * nx, rL * uLy * unL + pL * ny, rL * uLz * unL + pL * nz,
                              (UL[4] + pL) * unL};
        if (SL >= 0.0)
            for (int v = 0; v < 5; ++v) F[v] = FL[v] * A;
        else
            star(UL, FL, rL, pL, uLx, uLy, uLz, unL, aL, SL, SM, nx, ny, nz, A, F);
    } else {
        const double FR[5] = {rR * unR, rR * uRx * unR + pR * nx, rR * uRy * unR + pR * ny, rR * uRz * unR + pR * nz,
                              (UR[4] + pR) * unR};
        if (SR <= 0.0)
            for (int v = 0; v < 5; ++v) F[v] = FR[v] * A;
        else
            star(UR, FR, rR, pR, uRx, uRy, uRz, unR, aR, SR, SM, nx, ny, nz, A, F);
    }
}

/* HllcFlux::analytical_physical_jacobian (fluxes/hllc.hpp:172-229). */
static void euler_jac(const oracle_solver* s, const double* U, double nx, double ny, double nz, double* J) {
    const double rho = U[0], u = U[1] / rho, v = U[2] / rho, w = U[3] / rho, E = U[4] / rho;
    const double p = pressure(s, U), g = s->gamma, ph = g - 1.0;
    const double un = u * nx + v * ny + w * nz, q2 = u * u + v * v + w * w, H = E + p / rho, h = 0.5 * ph * q2;
    const double Jv[25] = {0.0, nx, ny, nz, 0.0,
                           h * nx - u * un, un + nx * (1.0 - ph) * u, u * ny - ph * nx * v, u * nz - ph * nx * w, ph * nx,
                           h * ny - v * un, v * nx - ph * ny * u, un + ny * (1.0 - ph) * v, v * nz - ph * ny * w, ph * ny,
                           h * nz - w * un, w * nx - ph * nz * u, w * ny - ph * nz * v, un + nz * (1.0 - ph) * w, ph * nz,
                           un * (h - H), H * nx - ph * u * un, H * ny - ph * v * un, H * nz - ph * w * un, g * un};
    memcpy(J, Jv, sizeof(Jv));
}

/* ---------------------------------------------------------------- viscous */
/* ViscousFlux::face_flux (fluxes/viscous.hpp:90-175): cell-centre states,
 * averaged gradients, over-relaxed normal derivative. */
static double viscous(const oracle_solver* s, int f, const double* qL, const double* qR, const double* gL,
                      const double* gR, double mutL, double mutR, double nx, double ny, double nz, double A,
                      double* Fv) {
    const double pf = 0.5 * (qL[0] + qR[0]), uf = 0.5 * (qL[1] + qR[1]), vf = 0.5 * (qL[2] + qR[2]);
    const double wf = 0.5 * (qL[3] + qR[3]), Tf = 0.5 * (qL[4] + qR[4]);
    const double mu_lam = sutherland(Tf);
    const double mu_t = 0.5 * (mutL + mutR);
    const double mu = mu_lam + mu_t;
    const double k = (mu_lam * s->cp) / s->cfg.prandtl + (mu_t * s->cp) / s->cfg.prandtl_turb;
    const double id = s->finv_d[f];
    const double cx = nx - s->fdx[f] * id, cy = ny - s->fdy[f] * id, cz = nz - s->fdz[f] * id;
    double g[12];
    for (int i = 0; i < 12; ++i) g[i] = 0.5 * (gL[i] + gR[i]);
    const double div = g[0] + g[4] + g[8];
    const double ttd = (2.0 / 3.0) * div;
    const double du = (qR[1] - qL[1]) * id + (g[0] * cx + g[1] * cy + g[2] * cz);
    const double dv = (qR[2] - qL[2]) * id + (g[3] * cx + g[4] * cy + g[5] * cz);
    const double dw = (qR[3] - qL[3]) * id + (g[6] * cx + g[7] * cy + g[8] * cz);
    const double dT = (qR[4] - qL[4]) * id + (g[9] * cx + g[10] * cy + g[11] * cz);
    const double tx = mu * (du + (g[0] * nx + g[3] * ny + g[6] * nz) - ttd * nx);
    const double ty = mu * (dv + (g[1] * nx + g[4] * ny + g[7] * nz) - ttd * ny);
    const double tz = mu * (dw + (g[2] * nx + g[5] * ny + g[8] * nz) - ttd * nz);
    const double qn = -k * dT;
    Fv[0] = 0.0;
    Fv[1] = -tx * A;
    Fv[2] = -ty * A;
    Fv[3] = -tz * A;
    Fv[4] = (-(uf * tx + vf * ty + wf * tz) + qn) * A;
    const double rho_f = pf / (s->R * Tf);
    return (4.0 / 3.0) * (mu / rho_f) * id * A;
}

/* ViscousFlux::face_flux_jacobian, thin layer (fluxes/viscous.hpp:280-360).
 * full != 0 (CFDG_JAC_THIN_LAYER): mu/d (I + n n^T / 3) on the velocity, and
 * wv / wt scale the velocity / temperature derivatives (2 on a no-slip wall
 * face for the mirrored ghost velocity / isothermal temperature). */
static void viscous_jac(const oracle_solver* s, int f, const double* qL, const double* qR, double mutL, double mutR,
                        double A, double* J, int full, double wv, double wt) {
    const double pf = 0.5 * (qL[0] + qR[0]), uf = 0.5 * (qL[1] + qR[1]), vf = 0.5 * (qL[2] + qR[2]);
    const double wf = 0.5 * (qL[3] + qR[3]), Tf = 0.5 * (qL[4] + qR[4]);
    const double rho = pf / (s->R * Tf), ir = 1.0 / rho, irc = 1.0 / (rho * s->cv);
    const double mu_lam = sutherland(Tf), mu_t = 0.5 * (mutL + mutR), mu = mu_lam + mu_t;
    const double k = (mu_lam * s->cp) / s->cfg.prandtl + (mu_t * s->cp) / s->cfg.prandtl_turb;
    const double Cm = mu * s->finv_d[f] * A, Cl = k * s->finv_d[f] * A;
    const double V2 = uf * uf + vf * vf + wf * wf;
    memset(J, 0, 25 * sizeof(double));
    if (!full) {
        J[5] = -Cm * uf * ir;
        J[6] = Cm * ir;
        J[10] = -Cm * vf * ir;
        J[12] = Cm * ir;
        J[15] = -Cm * wf * ir;
        J[18] = Cm * ir;
        J[20] = Cl * (0.5 * V2 - s->cv * Tf) * irc - Cm * V2 * ir;
        J[21] = -Cl * uf * irc + Cm * uf * ir;
        J[22] = -Cl * vf * irc + Cm * vf * ir;
        J[23] = -Cl * wf * irc + Cm * wf * ir;
        J[24] = Cl * irc;
        return;
    }
    const double n[3] = {s->m.face_normal_x[f], s->m.face_normal_y[f], s->m.face_normal_z[f]};
    const double u[3] = {uf, vf, wf};
    const double cm = wv * Cm, cl = wt * Cl;
    double M[3][3], Mu[3] = {0, 0, 0};
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            M[a][b] = (a == b ? 1.0 : 0.0) + n[a] * n[b] / 3.0;
            Mu[a] += M[a][b] * u[b];
        }
    double uMu = 0.0;
    for (int a = 0; a < 3; ++a) {
        J[(1 + a) * 5] = -cm * Mu[a] * ir;
        for (int b = 0; b < 3; ++b) J[(1 + a) * 5 + 1 + b] = cm * M[a][b] * ir;
        uMu += u[a] * Mu[a];
    }
    J[20] = cl * (0.5 * V2 - s->cv * Tf) * irc - cm * uMu * ir;
    for (int b = 0; b < 3; ++b) J[21 + b] = -cl * u[b] * irc + cm * Mu[b] * ir;
    J[24] = cl * irc;
}

/* --------------------------------------------------------------- BCs */
/* compute_riemann_farfield_state (bc/physical/farfield.hpp:39-100). */
static int farfield(const oracle_solver* s, const bcp_t* P, const double* qi, double nx, double ny, double nz,
                    double* qb) {
    const double g = s->gamma, R = s->R, gm1 = g - 1.0;
    const double un_in = qi[1] * nx + qi[2] * ny + qi[3] * nz;
    const double un_inf = P->far_u * nx + P->far_v * ny + P->far_w * nz;
    const double a_in = sqrt(g * R * fmax(qi[4], 1e-6)), a_inf = sqrt(g * R * fmax(P->far_T, 1e-6));
    const double mn = un_in / a_in;
    if (mn >= 1.0) {
        memcpy(qb, qi, 5 * sizeof(double));
        return 1;
    }
    if (mn <= -1.0) {
        qb[0] = P->far_p;
        qb[1] = P->far_u;
        qb[2] = P->far_v;
        qb[3] = P->far_w;
        qb[4] = P->far_T;
        return 0;
    }
    const double Ro = un_in + 2.0 * a_in / gm1, Ri = un_inf - 2.0 * a_inf / gm1;
    const double unb = 0.5 * (Ro + Ri);
    double ab = 0.25 * gm1 * (Ro - Ri);
    if (ab <= 0.0) ab = a_inf;
    double ent;
    if (unb >= 0.0) {
        qb[1] = qi[1] + (unb - un_in) * nx;
        qb[2] = qi[2] + (unb - un_in) * ny;
        qb[3] = qi[3] + (unb - un_in) * nz;
        const double rin = qi[0] / (R * fmax(qi[4], 1e-6));
        ent = qi[0] / pow(fmax(rin, 1e-12), g);
    } else {
        qb[1] = P->far_u + (unb - un_inf) * nx;
        qb[2] = P->far_v + (unb - un_inf) * ny;
        qb[3] = P->far_w + (unb - un_inf) * nz;
        const double rinf = P->far_p / (R * fmax(P->far_T, 1e-6));
        ent = P->far_p / pow(fmax(rinf, 1e-12), g);
    }
    const double rb = pow(ab * ab / (g * fmax(ent, 1e-12)), 1.0 / gm1);
    qb[0] = rb * ab * ab / g;
    qb[4] = ab * ab / (g * R);
    return 0;
}

/* update_ghost_cells of the nine BC classes (bc/physical/*.hpp,
 * numerics/boundary/boundary_values.hpp). */
static void ghost_values(const oracle_solver* s, const bcp_t* P, const double* qi, double nx, double ny, double nz,
                         double rcfn, double* qg) {
    switch (P->kind) {
        case CFDG_BC_SUPERSONIC_INLET:
            for (int v = 0; v < 5; ++v) qg[v] = 2.0 * P->qfix[v] - qi[v];
            qg[0] = fmax(qg[0], 1.0);
            qg[4] = fmax(qg[4], 1.0);
            break;
        case CFDG_BC_SLIP_WALL:
        case CFDG_BC_SYMMETRY: {
            const double vn2 = 2.0 * (qi[1] * nx + qi[2] * ny + qi[3] * nz);
            qg[0] = qi[0];
            qg[1] = qi[1] - vn2 * nx;
            qg[2] = qi[2] - vn2 * ny;
            qg[3] = qi[3] - vn2 * nz;
            qg[4] = qi[4];
            break;
        }
        case CFDG_BC_FARFIELD: {
            double qb[5];
            if (farfield(s, P, qi, nx, ny, nz, qb)) {
                memcpy(qg, qi, 5 * sizeof(double));
            } else {
                for (int v = 0; v < 5; ++v) qg[v] = 2.0 * qb[v] - qi[v];
                qg[0] = fmax(qg[0], 1.0);
                qg[4] = fmax(qg[4], 1.0);
            }
            break;
        }
        case CFDG_BC_NO_SLIP_WALL:
        case CFDG_BC_SUBSONIC_INLET:
            qg[0] = qi[0];
            for (int v = 1; v < 5; ++v) qg[v] = 2.0 * P->qfix[v] - qi[v];
            qg[4] = fmax(qg[4], 1.0);
            break;
        case CFDG_BC_NO_SLIP_WALL_HEAT_FLUX: {
            qg[0] = qi[0];
            for (int v = 1; v < 4; ++v) qg[v] = 2.0 * P->qfix[v] - qi[v];
            const double r = 1.0 / (1.0 / fmax(rcfn, 1e-14));
            qg[4] = fmax(qi[4] + 2.0 * P->tmp_grad * r, 1.0);
            break;
        }
        case CFDG_BC_SUBSONIC_OUTLET:
            qg[0] = fmax(2.0 * P->p_out - qi[0], 1.0);
            for (int v = 1; v < 5; ++v) qg[v] = qi[v];
            break;
        default:
            memcpy(qg, qi, 5 * sizeof(double));
            break;
    }
}

/* numerics/boundary/boundary_gradients.hpp:15-160. */
static void g_dir(const double* gi, double qin, double qfix, double nx, double ny, double nz, double ri, double* gg) {
    const double f = 2.0 * ((qfix - qin) * ri - (gi[0] * nx + gi[1] * ny + gi[2] * nz));
    gg[0] = gi[0] + f * nx;
    gg[1] = gi[1] + f * ny;
    gg[2] = gi[2] + f * nz;
}
static void g_neu(const double* gi, double fixed, double nx, double ny, double nz, double* gg) {
    const double f = 2.0 * (fixed - (gi[0] * nx + gi[1] * ny + gi[2] * nz));
    gg[0] = gi[0] + f * nx;
    gg[1] = gi[1] + f * ny;
    gg[2] = gi[2] + f * nz;
}
static void g_slip(const double* gi, double qin, double qgh, double nx, double ny, double nz, double ri, double* gg) {
    const double gdn = gi[0] * nx + gi[1] * ny + gi[2] * nz;
    const double f = 2.0 * (0.5 * (qgh - qin) * ri - gdn);
    gg[0] = gi[0] + f * nx;
    gg[1] = gi[1] + f * ny;
    gg[2] = gi[2] + f * nz;
}

/* ---------------------------------------------------------------- setup */
static void resolve(const oracle_solver* s, const cfdg_bc_desc* d, double p_ref, double* out /* p u v w T */) {
    out[0] = p_ref;
    out[4] = d->t;
    if (d->inflow_mode == CFDG_INFLOW_VELOCITY) {
        out[1] = d->velocity[0];
        out[2] = d->velocity[1];
        out[3] = d->velocity[2];
        return;
    }
    const double rho = p_ref / (s->R * d->t);
    const double vm = d->mach * sqrt(s->gamma * p_ref / rho);
    if (d->inflow_mode == CFDG_INFLOW_MACH_ANGLES) {
        const double k = ORACLE_PI / 180.0, a = d->alpha_deg * k, b = d->beta_deg * k;
        out[1] = vm * cos(a) * cos(b);
        out[2] = -vm * sin(b);
        out[3] = vm * sin(a) * cos(b);
    } else {
        const double nr = sqrt(d->direction[0] * d->direction[0] + d->direction[1] * d->direction[1] +
                               d->direction[2] * d->direction[2]);
        const double inv = nr > 1e-14 ? 1.0 / nr : 0.0;
        out[1] = vm * d->direction[0] * inv;
        out[2] = vm * d->direction[1] * inv;
        out[3] = vm * d->direction[2] * inv;
    }
}

/* LeastSquaresCell{Face,Node}Gradient::setup (gradient_operator.cpp:414-499,
 * 622-707) with invert3x3 (:20-47). */
static void lsq_setup(oracle_solver* s) {
    const cfdg_mesh_host* m = &s->m;
    for (int c = 0; c < s->n; ++c) {
        const int p1 = s->g_off[c], p2 = s->g_off[c + 1];
        double A[9] = {0};
        for (int j = p1; j < p2; ++j) {
            const int nb = s->g_col[j];
            const double dx = m->cell_centroid_x[nb] - m->cell_centroid_x[c];
            const double dy = m->cell_centroid_y[nb] - m->cell_centroid_y[c];
            const double dz = m->cell_centroid_z[nb] - m->cell_centroid_z[c];
            const double w = 1.0 / fmax(dx * dx + dy * dy + dz * dz, 1e-30);
            A[0] += w * dx * dx;
            A[1] += w * dx * dy;
            A[2] += w * dx * dz;
            A[4] += w * dy * dy;
            A[5] += w * dy * dz;
            A[8] += w * dz * dz;
        }
        A[3] = A[1];
        A[6] = A[2];
        A[7] = A[5];
        A[0] += 1e-14;
        A[4] += 1e-14;
        A[8] += 1e-14;
        double I[9] = {0};
        const double det = A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
                           A[2] * (A[3] * A[7] - A[4] * A[6]);
        if (fabs(det) > 1e-14) {
            const double id = 1.0 / det;
            I[0] = (A[4] * A[8] - A[5] * A[7]) * id;
            I[1] = (A[2] * A[7] - A[1] * A[8]) * id;
            I[2] = (A[1] * A[5] - A[2] * A[4]) * id;
            I[3] = (A[5] * A[6] - A[3] * A[8]) * id;
            I[4] = (A[0] * A[8] - A[2] * A[6]) * id;
            I[5] = (A[2] * A[3] - A[0] * A[5]) * id;
            I[6] = (A[3] * A[7] - A[4] * A[6]) * id;
            I[7] = (A[1] * A[6] - A[0] * A[7]) * id;
            I[8] = (A[0] * A[4] - A[1] * A[3]) * id;
        }
        for (int j = p1; j < p2; ++j) {
            const int nb = s->g_col[j];
            const double dx = m->cell_centroid_x[nb] - m->cell_centroid_x[c];
            const double dy = m->cell_centroid_y[nb] - m->cell_centroid_y[c];
            const double dz = m->cell_centroid_z[nb] - m->cell_centroid_z[c];
            const double w = 1.0 / fmax(dx * dx + dy * dy + dz * dz, 1e-30);
            const double rx = w * dx, ry = w * dy, rz = w * dz;
            s->g_wx[j] = I[0] * rx + I[1] * ry + I[2] * rz;
            s->g_wy[j] = I[3] * rx + I[4] * ry + I[5] * rz;
            s->g_wz[j] = I[6] * rx + I[7] * ry + I[8] * rz;
        }
    }
}

/* MeshAuxGeometry::add_wall_distance with the face-neighbour stencil
 * (src/mesh/aux_geometry.cpp:541-696): seed wall-adjacent cells with the
 * owner-to-face-centroid distance, then forward/backward Gauss-Seidel
 * relaxation d_c = min(d_c, d_j + |x_c - x_j|) until the largest relative
 * change is <= tol or max_sweeps passes. */
static void wall_distance(oracle_solver* s, int max_sweeps, double tol) {
    const cfdg_mesh_host* m = &s->m;
    const int n = s->n;
    for (int c = 0; c < n; ++c) s->dist[c] = 1.0e30;
    for (int f = s->ni; f < s->nf; ++f) {
        if (s->bcp[m->face_patch[f]].sa_kind != 0) continue;
        const int c0 = m->face_owner[f];
        const double ex = m->face_centroid_x[f] - m->cell_centroid_x[c0];
        const double ey = m->face_centroid_y[f] - m->cell_centroid_y[c0];
        const double ez = m->face_centroid_z[f] - m->cell_centroid_z[c0];
        const double d = sqrt(ex * ex + ey * ey + ez * ez);
        if (d < s->dist[c0]) s->dist[c0] = d;
    }
    for (int sweep = 0; sweep < max_sweeps; ++sweep) {
        double max_rel = 0.0;
        for (int pass = 0; pass < 2; ++pass)
            for (int k = 0; k < n; ++k) {
                const int c = pass == 0 ? k : n - 1 - k;
                const double d0 = s->dist[c];
                double dn = d0;
                for (int j = s->c2c_off[c]; j < s->c2c_off[c + 1]; ++j) {
                    const int o = s->c2c[j];
                    const double dx = m->cell_centroid_x[o] - m->cell_centroid_x[c];
                    const double dy = m->cell_centroid_y[o] - m->cell_centroid_y[c];
                    const double dz = m->cell_centroid_z[o] - m->cell_centroid_z[c];
                    const double cand = s->dist[o] + sqrt(dx * dx + dy * dy + dz * dz);
                    dn = cand < dn ? cand : dn;
                }
                if (dn < d0) {
                    const double rel = (d0 - dn) / (d0 > 1.0e-12 ? d0 : 1.0e-12);
                    if (rel > max_rel) max_rel = rel;
                    s->dist[c] = dn;
                }
            }
        if (max_rel <= tol) break;
    }
}

int oracle_create(const cfdg_mesh_host* m, const cfdg_config* cfg, const cfdg_bc_desc* bcs, int nbc,
                  oracle_solver** out) {
    oracle_solver* s = (oracle_solver*)calloc(1, sizeof(oracle_solver));
    s->m = *m;
    s->cfg = *cfg;
    s->gamma = cfg->gamma;
    s->R = cfg->gas_constant;
    s->cv = s->R / (s->gamma - 1.0);
    s->cp = s->gamma * s->cv;
    s->n = m->n_cells;
    s->nf = m->n_faces;
    s->ni = m->n_inner_faces;
    s->nb = s->nf - s->ni;
    s->nt = s->n + s->nb;
    s->sa = cfg->turbulence == 1;
    s->nv = s->sa ? 6 : 5;
    s->muscl = cfg->reconstruction == CFDG_RECON_MUSCL;
    s->visc = cfg->viscous != 0;
    s->need_grad = s->muscl || s->visc;
    s->n_patch = m->n_patches > 0 ? m->n_patches : 1;
    s->bcp = (bcp_t*)xcalloc((size_t)s->n_patch, sizeof(bcp_t));
    for (int p = 0; p < s->n_patch; ++p) {
        s->bcp[p].kind = -1;
        s->bcp[p].sa_kind = 3;
    }
    /* BoundaryManager::register_all parameter resolution (bc_manager.hpp:223-329) */
    for (int i = 0; i < nbc; ++i) {
        const cfdg_bc_desc* d = &bcs[i];
        if (d->patch_id < 0 || d->patch_id >= s->n_patch) continue;
        bcp_t* P = &s->bcp[d->patch_id];
        memset(P, 0, sizeof(*P));
        P->kind = d->type;
        /* SpalartAllmaras::zone_kind (spalart_allmaras.hpp:458-475) */
        switch (d->type) {
            case CFDG_BC_NO_SLIP_WALL:
            case CFDG_BC_NO_SLIP_WALL_HEAT_FLUX: P->sa_kind = 0; break;
            case CFDG_BC_SUPERSONIC_INLET:
            case CFDG_BC_SUBSONIC_INLET:
            case CFDG_BC_FARFIELD: P->sa_kind = 1; break;
            case CFDG_BC_SUPERSONIC_OUTLET:
            case CFDG_BC_SUBSONIC_OUTLET: P->sa_kind = 2; break;
            default: P->sa_kind = 3; break;
        }
        double st[5];
        switch (d->type) {
            case CFDG_BC_SUPERSONIC_INLET:
                resolve(s, d, d->p, st);
                memcpy(P->qfix, st, sizeof(st));
                break;
            case CFDG_BC_FARFIELD:
                resolve(s, d, d->p, st);
                P->far_p = st[0];
                P->far_u = st[1];
                P->far_v = st[2];
                P->far_w = st[3];
                P->far_T = st[4];
                break;
            case CFDG_BC_NO_SLIP_WALL:
                P->qfix[1] = d->velocity[0];
                P->qfix[2] = d->velocity[1];
                P->qfix[3] = d->velocity[2];
                P->qfix[4] = d->t;
                break;
            case CFDG_BC_NO_SLIP_WALL_HEAT_FLUX:
                P->qfix[1] = d->velocity[0];
                P->qfix[2] = d->velocity[1];
                P->qfix[3] = d->velocity[2];
                P->tmp_grad = d->tmp_grad;
                break;
            case CFDG_BC_SUBSONIC_INLET:
                resolve(s, d, d->p > 0.0 ? d->p : 101325.0, st);
                memcpy(P->qfix, st, sizeof(st));
                break;
            case CFDG_BC_SUBSONIC_OUTLET:
                P->p_out = d->p;
                break;
            default:
                break;
        }
    }
    const int n = s->n;
    /* connectivity */
    s->c2f_off = (int32_t*)xcalloc((size_t)n + 1, 4);
    s->c2f = (int32_t*)xcalloc((size_t)oracle_connectivity(m, 0, NULL, NULL), 4);
    oracle_connectivity(m, 0, s->c2f_off, s->c2f);
    s->c2c_off = (int32_t*)xcalloc((size_t)n + 1, 4);
    s->c2c = (int32_t*)xcalloc((size_t)oracle_connectivity(m, 1, NULL, NULL), 4);
    oracle_connectivity(m, 1, s->c2c_off, s->c2c);
    const int gk = (cfg->gradient == CFDG_GRAD_LSQ_FACE) ? 1 : 2;
    s->g_off = (int32_t*)xcalloc((size_t)n + 1, 4);
    const int64_t ge = oracle_connectivity(m, gk, s->g_off, NULL);
    s->g_col = (int32_t*)xcalloc((size_t)ge, 4);
    oracle_connectivity(m, gk, s->g_off, s->g_col);
    s->g_wx = (double*)xcalloc((size_t)ge, 8);
    s->g_wy = (double*)xcalloc((size_t)ge, 8);
    s->g_wz = (double*)xcalloc((size_t)ge, 8);
    lsq_setup(s);
    /* face-cell distance vectors (aux_geometry.cpp:11-51, 107-156) */
    s->fdx = (double*)xcalloc((size_t)s->nf, 8);
    s->fdy = (double*)xcalloc((size_t)s->nf, 8);
    s->fdz = (double*)xcalloc((size_t)s->nf, 8);
    s->finv_d = (double*)xcalloc((size_t)s->nf, 8);
    for (int f = 0; f < s->nf; ++f) {
        const int u = m->face_owner[f];
        if (f < s->ni) {
            const int v = m->face_neigh[f];
            s->fdx[f] = m->cell_centroid_x[v] - m->cell_centroid_x[u];
            s->fdy[f] = m->cell_centroid_y[v] - m->cell_centroid_y[u];
            s->fdz[f] = m->cell_centroid_z[v] - m->cell_centroid_z[u];
        } else {
            s->fdx[f] = 2.0 * (m->face_centroid_x[f] - m->cell_centroid_x[u]);
            s->fdy[f] = 2.0 * (m->face_centroid_y[f] - m->cell_centroid_y[u]);
            s->fdz[f] = 2.0 * (m->face_centroid_z[f] - m->cell_centroid_z[u]);
        }
        s->finv_d[f] = 1.0 / sqrt(s->fdx[f] * s->fdx[f] + s->fdy[f] * s->fdy[f] + s->fdz[f] * s->fdz[f]);
    }
    /* BSR structure (bsr_helpers.hpp:16-59) */
    s->rp = (int32_t*)xcalloc((size_t)n + 1, 4);
    for (int c = 0; c < n; ++c) s->rp[c + 1] = s->rp[c] + 1 + (s->c2c_off[c + 1] - s->c2c_off[c]);
    s->nnzb = s->rp[n];
    s->cols = (int32_t*)xcalloc((size_t)s->nnzb, 4);
    s->diag = (int32_t*)xcalloc((size_t)n, 4);
    for (int c = 0; c < n; ++c) {
        int w = s->rp[c];
        s->cols[w++] = c;
        for (int k = s->c2c_off[c]; k < s->c2c_off[c + 1]; ++k) s->cols[w++] = s->c2c[k];
        qsort(s->cols + s->rp[c], (size_t)(s->rp[c + 1] - s->rp[c]), 4, cmp_i32);
        for (int k = s->rp[c]; k < s->rp[c + 1]; ++k)
            if (s->cols[k] == c) s->diag[c] = k;
    }
    const size_t nt = (size_t)s->nt, nv = (size_t)s->nv;
    s->U = (double*)xcalloc(nv * (size_t)n, 8);
    s->q = (double*)xcalloc(5 * nt, 8);
    s->grad = (double*)xcalloc(15 * nt, 8);
    s->phi = (double*)xcalloc(5 * (size_t)n, 8);
    s->res = (double*)xcalloc(nv * (size_t)n, 8);
    s->lam = (double*)xcalloc((size_t)n, 8);
    s->alpha = (double*)xcalloc((size_t)n, 8);
    s->vals = (double*)xcalloc((size_t)s->nnzb * nv * nv, 8);
    if (s->sa) {
        s->dist = (double*)xcalloc((size_t)n, 8);
        s->nu = (double*)xcalloc(nt, 8);
        s->rho = (double*)xcalloc(nt, 8);
        s->mut = (double*)xcalloc(nt, 8);
        s->gnu = (double*)xcalloc(3 * nt, 8);
        s->mdot = (double*)xcalloc((size_t)s->nf, 8);
        s->rhonu_g = (double*)xcalloc((size_t)s->nb, 8);
        wall_distance(s, 1000000, 0.0); /* to the exact graph fixed point */
        /* SpalartAllmaras::initialize freestream values (spalart_allmaras.hpp:193-198) */
        const double T_inf = cfg->init_p / (cfg->init_rho * s->R);
        s->nu_inf = cfg->nu_inf_ratio * sutherland(T_inf) / cfg->init_rho;
        s->rhonu_inf = cfg->init_rho * s->nu_inf;
    }
    *out = s;
    return 0;
}

void oracle_destroy(oracle_solver* s) {
    if (!s) return;
    void* p[] = {s->bcp, s->c2f_off, s->c2f, s->c2c_off, s->c2c, s->g_off, s->g_col, s->g_wx, s->g_wy, s->g_wz,
                 s->fdx, s->fdy, s->fdz, s->finv_d, s->rp, s->cols, s->diag, s->U, s->q, s->grad, s->phi, s->res,
                 s->lam, s->alpha, s->vals, s->dist, s->nu, s->rho, s->mut, s->gnu, s->mdot, s->rhonu_g};
    for (size_t i = 0; i < sizeof(p) / sizeof(p[0]); ++i) free(p[i]);
    free(s);
}

int64_t oracle_nnzb(const oracle_solver* s) { return s->nnzb; }
int oracle_nvars(const oracle_solver* s) { return s->nv; }

int oracle_structure(const oracle_solver* s, int32_t* row_ptr, int32_t* cols) {
    memcpy(row_ptr, s->rp, sizeof(int32_t) * ((size_t)s->n + 1));
    memcpy(cols, s->cols, sizeof(int32_t) * (size_t)s->nnzb);
    return 0;
}

void oracle_set_state(oracle_solver* s, const double* U, int64_t ld) {
    for (int v = 0; v < s->nv; ++v) memcpy(s->U + (size_t)v * s->n, U + v * ld, sizeof(double) * (size_t)s->n);
}

void oracle_get_state(const oracle_solver* s, double* U, int64_t ld) {
    for (int v = 0; v < s->nv; ++v) memcpy(U + v * ld, s->U + (size_t)v * s->n, sizeof(double) * (size_t)s->n);
}

/* Averaged + skew-corrected nu_tilde face gradient
 * (SpalartAllmaras::face_gradient, spalart_allmaras.hpp:486-508). */
static void sa_face_gradient(const oracle_solver* s, int f, int cl, double nul, int cr, double nur, double* gn) {
    const size_t nt = (size_t)s->nt;
    const double dx = s->fdx[f], dy = s->fdy[f], dz = s->fdz[f];
    gn[0] = 0.5 * (s->gnu[cl] + s->gnu[cr]);
    gn[1] = 0.5 * (s->gnu[nt + cl] + s->gnu[nt + cr]);
    gn[2] = 0.5 * (s->gnu[2 * nt + cl] + s->gnu[2 * nt + cr]);
    const double gd = gn[0] * dx + gn[1] * dy + gn[2] * dz;
    const double id = s->finv_d[f];
    const double corr = ((nur - nul) - gd) * id * id;
    gn[0] += corr * dx;
    gn[1] += corr * dy;
    gn[2] += corr * dz;
}

/* Spalart-Allmaras convection + diffusion face sweep and cell sources
 * (SpalartAllmaras::face_sweep / cell_sources, spalart_allmaras.hpp:291-432)
 * with the standard SA-1994 signs: the diffusive flux enters the residual
 * with a minus sign (the reference adds it), the cb2 term is a source
 * (the reference adds it to the residual), S = sqrt(2 S_ij S_ij) with full
 * weight on the shear terms (the reference halves them) and
 * f_w = g ((1 + cw3^6) / (g^6 + cw3^6))^(1/6) (the reference drops cw3^6
 * from the denominator); at walls and symmetry planes the boundary face is
 * never an inflow (the reference tests the sign of a round-off mass flux). */
/* f_w of cell c from the stored nu_tilde, wall distance and gradients. */
static double sa_fw_core(const oracle_solver* s, int c, double* sbar_out) {
    const size_t nt = (size_t)s->nt;
    const double rho = s->rho[c], nu = s->nu[c];
    const double d = fmax(s->dist[c], SA_MIN_WALL_DIST), id2 = 1.0 / (d * d);
    const double* gr = s->grad;
    const double ux = gr[3 * nt + c], uy = gr[4 * nt + c], uz = gr[5 * nt + c];
    const double vx = gr[6 * nt + c], vy = gr[7 * nt + c], vz = gr[8 * nt + c];
    const double wx = gr[9 * nt + c], wy = gr[10 * nt + c], wz = gr[11 * nt + c];
    const double sxy = uy + vx, sxz = uz + wx, syz = vz + wy;
    const double s2 = 2.0 * (ux * ux + vy * vy + wz * wz) + sxy * sxy + sxz * sxz + syz * syz;
    const double S = sqrt(fmax(s2, 0.0));
    const double nu_lam = sutherland(s->q[4 * nt + c]) / rho;
    const double chi = nu / nu_lam, chi3 = chi * chi * chi;
    const double fv1 = chi3 / (chi3 + SA_CV1 * SA_CV1 * SA_CV1);
    const double fv2 = 1.0 - chi / (1.0 + chi * fv1);
    const double ik2 = 1.0 / (SA_KAPPA * SA_KAPPA);
    const double sbar = fmax(S + nu * fv2 * ik2 * id2, SA_SBAR_FLOOR);
    double r = nu / (sbar * SA_KAPPA * SA_KAPPA * d * d);
    r = fmin(fmax(r, 0.0), 10.0);
    const double r2 = r * r, r6 = r2 * r2 * r2;
    const double g = r + SA_CW2 * (r6 - r);
    const double g2 = g * g, g6 = g2 * g2 * g2;
    const double cw3_6 = SA_CW3 * SA_CW3 * SA_CW3 * SA_CW3 * SA_CW3 * SA_CW3;
    if (sbar_out) *sbar_out = sbar;
    return g * pow((1.0 + cw3_6) / (g6 + cw3_6), 1.0 / 6.0);
}

static double sa_fw(const oracle_solver* s, int c) { return sa_fw_core(s, c, NULL); }

static void sa_residual(oracle_solver* s) {
    const cfdg_mesh_host* m = &s->m;
    const int n = s->n, nt = s->nt, ni = s->ni, nf = s->nf;
    double* res = s->res + (size_t)5 * n;
    const double is = 1.0 / SA_SIGMA;
    memset(res, 0, sizeof(double) * (size_t)n);
    for (int f = 0; f < nf; ++f) {
        const int inner = f < ni;
        const int c0 = m->face_owner[f], b = f - ni;
        const int c1 = inner ? m->face_neigh[f] : n + b;
        const double nx = m->face_normal_x[f], ny = m->face_normal_y[f], nz = m->face_normal_z[f], A = m->face_area[f];
        const double mf = s->mdot[f];
        double gn[3];
        if (inner) {
            const double nu_up = (mf >= 0.0) ? s->nu[c0] : s->nu[c1];
            sa_face_gradient(s, f, c0, s->nu[c0], c1, s->nu[c1], gn);
            const double Tf = 0.5 * (s->q[4 * (size_t)nt + c0] + s->q[4 * (size_t)nt + c1]);
            const double mu_f = sutherland(Tf);
            const double rho_f = 0.5 * (s->rho[c0] + s->rho[c1]);
            const double nu_f = 0.5 * (s->nu[c0] + s->nu[c1]);
            const double coef = is * (mu_f + rho_f * nu_f);
            const double fd = coef * (gn[0] * nx + gn[1] * ny + gn[2] * nz) * A;
            const double flux = mf * nu_up - fd;
            res[c0] += flux;
            res[c1] -= flux;
            const double w = fabs(mf) / rho_f + 2.0 * is * (mu_f + rho_f * nu_f) / rho_f * A * s->finv_d[f];
            s->lam[c0] += w;
            s->lam[c1] += w;
        } else {
            /* walls and symmetry planes carry no mass flux: their m is
             * round-off, so only inflow/outflow patches switch on its sign */
            const int kind = s->bcp[m->face_patch[f]].sa_kind;
            const int inflow = (kind == 1 || kind == 2) && mf < 0.0;
            const double pg = s->q[0 * (size_t)nt + c1], Tg = s->q[4 * (size_t)nt + c1];
            const double rho_g = pg / (s->R * Tg);
            const double nu_g = inflow ? s->nu_inf : s->rhonu_g[b] / rho_g;
            const double nu_up = inflow ? s->nu_inf : s->nu[c0];
            sa_face_gradient(s, f, c0, s->nu[c0], c1, nu_g, gn);
            const double Tf = 0.5 * (s->q[4 * (size_t)nt + c0] + Tg);
            const double mu_f = sutherland(Tf);
            const double rho_f = 0.5 * (s->rho[c0] + rho_g);
            const double coef = is * (mu_f + rho_f * 0.5 * (s->nu[c0] + nu_g));
            const double fd = coef * (gn[0] * nx + gn[1] * ny + gn[2] * nz) * A;
            res[c0] += mf * nu_up - fd;
        }
    }
    for (int c = 0; c < n; ++c) {
        const double rho = s->rho[c], nu = s->nu[c];
        const double d = fmax(s->dist[c], SA_MIN_WALL_DIST), id2 = 1.0 / (d * d);
        double sbar;
        const double fw = sa_fw_core(s, c, &sbar);
        const double P = SA_CB1 * sbar * rho * nu;
        const double D = SA_CW1 * fw * rho * nu * nu * id2;
        const double gnx = s->gnu[c], gny = s->gnu[(size_t)nt + c], gnz = s->gnu[2 * (size_t)nt + c];
        const double cb2 = (SA_CB2 / SA_SIGMA) * rho * (gnx * gnx + gny * gny + gnz * gnz);
        res[c] += m->cell_volume[c] * (D - P - cb2);
    }
}

/* ------------------------------------------------------- residual pipeline */
/* Solver::evaluate_residual steps 1-6 (solver.hpp:169-247). */
static void residual(oracle_solver* s) {
    const cfdg_mesh_host* m = &s->m;
    const int n = s->n, nt = s->nt, ni = s->ni, nf = s->nf;
    double* q = s->q;
    /* 1: conserved -> primitive */
    for (int c = 0; c < n; ++c) {
        const double U[5] = {s->U[c], s->U[n + c], s->U[2 * n + c], s->U[3 * n + c], s->U[4 * n + c]};
        double qc[5];
        cons2prim(s, U, qc);
        for (int v = 0; v < 5; ++v) q[v * nt + c] = qc[v];
    }
    /* 3: BC ghosts */
    for (int f = ni; f < nf; ++f) {
        const int c0 = m->face_owner[f], g = n + (f - ni);
        const double nx = m->face_normal_x[f], ny = m->face_normal_y[f], nz = m->face_normal_z[f];
        const double rcfn = (m->face_centroid_x[f] - m->cell_centroid_x[c0]) * nx +
                            (m->face_centroid_y[f] - m->cell_centroid_y[c0]) * ny +
                            (m->face_centroid_z[f] - m->cell_centroid_z[c0]) * nz;
        double qi[5], qg[5];
        for (int v = 0; v < 5; ++v) qi[v] = q[v * nt + c0];
        ghost_values(s, &s->bcp[m->face_patch[f]], qi, nx, ny, nz, rcfn, qg);
        for (int v = 0; v < 5; ++v) q[v * nt + g] = qg[v];
    }
    if (s->sa) {
        /* SpalartAllmaras::apply_bcs (spalart_allmaras.hpp:234-257): ghost rho*nu_tilde */
        for (int f = ni; f < nf; ++f) {
            const int c0 = m->face_owner[f], b = f - ni, g = n + b;
            const bcp_t* P = &s->bcp[m->face_patch[f]];
            const double rn0 = s->U[(size_t)5 * n + c0];
            if (P->sa_kind == 0) s->rhonu_g[b] = -rn0;
            else if (P->sa_kind == 1) s->rhonu_g[b] = (q[0 * nt + g] / (s->R * q[4 * nt + g])) * s->nu_inf;
            else s->rhonu_g[b] = rn0;
        }
        /* SpalartAllmaras::pre_sweep (spalart_allmaras.hpp:263-282): density,
         * specific nu_tilde and eddy viscosity on cells; zero eddy viscosity on
         * BC ghosts */
        for (int c = 0; c < n; ++c) {
            const double rho = q[0 * nt + c] / (s->R * q[4 * nt + c]);
            const double nu = s->U[(size_t)5 * n + c] / rho;
            s->rho[c] = rho;
            s->nu[c] = nu;
            const double nu_lam = sutherland(q[4 * nt + c]) / rho;
            const double chi = nu / nu_lam, chi3 = chi * chi * chi;
            const double fv1 = chi3 / (chi3 + SA_CV1 * SA_CV1 * SA_CV1);
            s->mut[c] = rho * nu * fv1;
        }
        for (int g = n; g < nt; ++g) {
            s->mut[g] = 0.0;
            s->rho[g] = 0.0;
            s->nu[g] = 0.0;
        }
    }
    if (s->need_grad) {
        /* 5: LSQ gradients (apply_kernel_lsq*, gradient_operator.cpp:340-391,549-599) */
        for (int c = 0; c < n; ++c) {
            double gx[5] = {0}, gy[5] = {0}, gz[5] = {0};
            for (int j = s->g_off[c]; j < s->g_off[c + 1]; ++j) {
                const int nb = s->g_col[j];
                for (int v = 0; v < 5; ++v) {
                    const double d = q[v * nt + nb] - q[v * nt + c];
                    gx[v] += s->g_wx[j] * d;
                    gy[v] += s->g_wy[j] * d;
                    gz[v] += s->g_wz[j] * d;
                }
            }
            for (int v = 0; v < 5; ++v) {
                s->grad[(3 * v + 0) * (size_t)nt + c] = gx[v];
                s->grad[(3 * v + 1) * (size_t)nt + c] = gy[v];
                s->grad[(3 * v + 2) * (size_t)nt + c] = gz[v];
            }
        }
        /* ghost gradients (update_ghost_cells_grad, bc/physical/*.hpp) */
        for (int f = ni; f < nf; ++f) {
            const int c0 = m->face_owner[f], g = n + (f - ni);
            const bcp_t* P = &s->bcp[m->face_patch[f]];
            const double nx = m->face_normal_x[f], ny = m->face_normal_y[f], nz = m->face_normal_z[f];
            const double rcfn = (m->face_centroid_x[f] - m->cell_centroid_x[c0]) * nx +
                                (m->face_centroid_y[f] - m->cell_centroid_y[c0]) * ny +
                                (m->face_centroid_z[f] - m->cell_centroid_z[c0]) * nz;
            const double ri = 1.0 / fmax(rcfn, 1e-14);
            double gi[5][3], gg[5][3], qi[5], qgh[5];
            for (int v = 0; v < 5; ++v) {
                qi[v] = q[v * nt + c0];
                qgh[v] = q[v * nt + g];
                for (int d = 0; d < 3; ++d) gi[v][d] = s->grad[(3 * v + d) * (size_t)nt + c0];
            }
            double qb[5];
            switch (P->kind) {
                case CFDG_BC_SUPERSONIC_INLET:
                    for (int v = 0; v < 5; ++v) g_dir(gi[v], qi[v], P->qfix[v], nx, ny, nz, ri, gg[v]);
                    break;
                case CFDG_BC_SLIP_WALL:
                case CFDG_BC_SYMMETRY:
                    g_neu(gi[0], 0.0, nx, ny, nz, gg[0]);
                    for (int v = 1; v < 4; ++v) g_slip(gi[v], qi[v], qgh[v], nx, ny, nz, ri, gg[v]);
                    g_neu(gi[4], 0.0, nx, ny, nz, gg[4]);
                    break;
                case CFDG_BC_FARFIELD:
                    if (farfield(s, P, qi, nx, ny, nz, qb))
                        memcpy(gg, gi, sizeof(gg));
                    else
                        for (int v = 0; v < 5; ++v) g_dir(gi[v], qi[v], qb[v], nx, ny, nz, ri, gg[v]);
                    break;
                case CFDG_BC_NO_SLIP_WALL:
                case CFDG_BC_SUBSONIC_INLET:
                    memcpy(gg[0], gi[0], sizeof(gg[0]));
                    for (int v = 1; v < 5; ++v) g_dir(gi[v], qi[v], P->qfix[v], nx, ny, nz, ri, gg[v]);
                    break;
                case CFDG_BC_NO_SLIP_WALL_HEAT_FLUX:
                    memcpy(gg[0], gi[0], sizeof(gg[0]));
                    for (int v = 1; v < 4; ++v) g_dir(gi[v], qi[v], P->qfix[v], nx, ny, nz, ri, gg[v]);
                    g_neu(gi[4], P->tmp_grad, nx, ny, nz, gg[4]);
                    break;
                case CFDG_BC_SUBSONIC_OUTLET:
                    g_dir(gi[0], qi[0], P->p_out, nx, ny, nz, ri, gg[0]);
                    for (int v = 1; v < 5; ++v) memcpy(gg[v], gi[v], sizeof(gg[v]));
                    break;
                default:
                    memcpy(gg, gi, sizeof(gg));
                    break;
            }
            for (int v = 0; v < 5; ++v)
                for (int d = 0; d < 3; ++d) s->grad[(3 * v + d) * (size_t)nt + g] = gg[v][d];
        }
    }
    if (s->sa) {
        /* nu_tilde gradient with the solver's least-squares stencil on cells,
         * BC ghost planes mirror the owner with a sign flip at walls
         * (SpalartAllmaras::compute_gradients, spalart_allmaras.hpp:212-229) */
        for (int c = 0; c < n; ++c) {
            double gx = 0, gy = 0, gz = 0;
            for (int j = s->g_off[c]; j < s->g_off[c + 1]; ++j) {
                const double d = s->nu[s->g_col[j]] - s->nu[c];
                gx += s->g_wx[j] * d;
                gy += s->g_wy[j] * d;
                gz += s->g_wz[j] * d;
            }
            s->gnu[c] = gx;
            s->gnu[(size_t)nt + c] = gy;
            s->gnu[2 * (size_t)nt + c] = gz;
        }
        for (int f = ni; f < nf; ++f) {
            const int c0 = m->face_owner[f], g = n + (f - ni);
            const double sg = (s->bcp[m->face_patch[f]].sa_kind == 0) ? -1.0 : 1.0;
            for (int p = 0; p < 3; ++p) s->gnu[(size_t)p * nt + g] = sg * s->gnu[(size_t)p * nt + c0];
        }
    }
    if (s->muscl && !s->phi_frozen) {
        /* Muscl::compute_limiters (numerics/reconstruction/muscl.hpp:25-105) */
        const double k3 = s->cfg.venkat_k * s->cfg.venkat_k * s->cfg.venkat_k;
        for (int c = 0; c < n; ++c) {
            double qc[5], qmax[5], qmin[5], ph[5];
            for (int v = 0; v < 5; ++v) {
                qc[v] = qmax[v] = qmin[v] = q[v * nt + c];
                ph[v] = 1.0;
            }
            for (int j = s->c2c_off[c]; j < s->c2c_off[c + 1]; ++j)
                for (int v = 0; v < 5; ++v) {
                    const double x = q[v * nt + s->c2c[j]];
                    qmax[v] = fmax(qmax[v], x);
                    qmin[v] = fmin(qmin[v], x);
                }
            const double eps2 = k3 * m->cell_volume[c];
            for (int e = s->c2f_off[c]; e < s->c2f_off[c + 1]; ++e) {
                const int f = s->c2f[e];
                const double ex = m->face_centroid_x[f] - m->cell_centroid_x[c];
                const double ey = m->face_centroid_y[f] - m->cell_centroid_y[c];
                const double ez = m->face_centroid_z[f] - m->cell_centroid_z[c];
                for (int v = 0; v < 5; ++v) {
                    const double df = s->grad[(3 * v) * (size_t)nt + c] * ex + s->grad[(3 * v + 1) * (size_t)nt + c] * ey +
                                      s->grad[(3 * v + 2) * (size_t)nt + c] * ez;
                    const double dnb = df > 0.0 ? qmax[v] - qc[v] : qmin[v] - qc[v];
                    double phv;
                    /* MultidimSlopeLimiter::phi (numerics/limiter/slope_limiters.hpp:21-79) */
                    if (df == 0.0) {
                        phv = 1.0;
                    } else if (s->cfg.limiter == CFDG_LIM_BARTH_JESPERSEN) {
                        phv = fmin(fmax(dnb / df, 0.0), 1.0);
                    } else if (dnb * df <= 0.0) {
                        phv = 0.0;
                    } else if (s->cfg.limiter == CFDG_LIM_VAN_ALBADA) {
                        const double den = dnb * dnb + df * df + eps2;
                        phv = den > 0.0 ? (dnb * dnb + dnb * df) / den : 1.0;
                    } else {
                        const double a2 = dnb * dnb + eps2;
                        phv = (a2 + 2.0 * dnb * df) / (a2 + 2.0 * df * df + dnb * df);
                    }
                    ph[v] = fmin(ph[v], phv);
                }
            }
            for (int v = 0; v < 5; ++v) s->phi[v * (size_t)n + c] = ph[v];
        }
    }
    /* 6: face sweep with sequential scatter (ResidualKernel::compute_fluxes,
     * residual_kernel.hpp:175-306) */
    memset(s->res, 0, sizeof(double) * 5 * (size_t)n);
    memset(s->lam, 0, sizeof(double) * (size_t)n);
    for (int f = 0; f < nf; ++f) {
        const int inner = f < ni;
        const int c0 = m->face_owner[f], c1 = inner ? m->face_neigh[f] : n + (f - ni);
        const double nx = m->face_normal_x[f], ny = m->face_normal_y[f], nz = m->face_normal_z[f], A = m->face_area[f];
        double qL[5], qR[5];
        for (int v = 0; v < 5; ++v) {
            qL[v] = q[v * nt + c0];
            qR[v] = q[v * nt + c1];
        }
        if (s->muscl && inner) {
            const double fx = m->face_centroid_x[f], fy = m->face_centroid_y[f], fz = m->face_centroid_z[f];
            for (int v = 0; v < 5; ++v) {
                const double d0 = s->grad[(3 * v) * (size_t)nt + c0] * (fx - m->cell_centroid_x[c0]) +
                                  s->grad[(3 * v + 1) * (size_t)nt + c0] * (fy - m->cell_centroid_y[c0]) +
                                  s->grad[(3 * v + 2) * (size_t)nt + c0] * (fz - m->cell_centroid_z[c0]);
                const double d1 = s->grad[(3 * v) * (size_t)nt + c1] * (fx - m->cell_centroid_x[c1]) +
                                  s->grad[(3 * v + 1) * (size_t)nt + c1] * (fy - m->cell_centroid_y[c1]) +
                                  s->grad[(3 * v + 2) * (size_t)nt + c1] * (fz - m->cell_centroid_z[c1]);
                qL[v] = q[v * nt + c0] + s->phi[v * (size_t)n + c0] * d0;
                qR[v] = q[v * nt + c1] + s->phi[v * (size_t)n + c1] * d1;
            }
        }
        double UL[5], UR[5], F[5], smax;
        prim2cons(s, qL, UL);
        prim2cons(s, qR, UR);
        hllc(s, UL, UR, nx, ny, nz, A, F, &smax);
        if (s->sa) s->mdot[f] = F[0];
        double lf = A * smax;
        if (s->visc) {
            double qcL[5], qcR[5], gL[12], gR[12], Fv[5];
            for (int v = 0; v < 5; ++v) {
                qcL[v] = q[v * nt + c0];
                qcR[v] = q[v * nt + c1];
            }
            for (int v = 1; v < 5; ++v)
                for (int d = 0; d < 3; ++d) {
                    gL[(v - 1) * 3 + d] = s->grad[(3 * v + d) * (size_t)nt + c0];
                    gR[(v - 1) * 3 + d] = s->grad[(3 * v + d) * (size_t)nt + c1];
                }
            const double mutL = s->sa ? s->mut[c0] : 0.0, mutR = s->sa ? s->mut[c1] : 0.0;
            lf += viscous(s, f, qcL, qcR, gL, gR, mutL, mutR, nx, ny, nz, A, Fv);
            for (int v = 1; v < 5; ++v) F[v] += Fv[v];
        }
        for (int v = 0; v < 5; ++v) {
            s->res[v * (size_t)n + c0] += F[v];
            if (inner) s->res[v * (size_t)n + c1] -= F[v];
        }
        s->lam[c0] += lf;
        if (inner) s->lam[c1] += lf;
    }
    if (s->sa) sa_residual(s);
}

void oracle_stages(oracle_solver* s, double* q, double* grad, double* phi, double* res, double* lam) {
    residual(s);
    const size_t n = (size_t)s->n, nt = (size_t)s->nt;
    if (q) memcpy(q, s->q, sizeof(double) * 5 * nt);
    if (grad) memcpy(grad, s->grad, sizeof(double) * 15 * nt);
    if (phi) memcpy(phi, s->phi, sizeof(double) * 5 * n);
    if (res) memcpy(res, s->res, sizeof(double) * (size_t)s->nv * n);
    if (lam) memcpy(lam, s->lam, sizeof(double) * n);
}

/* ------------------------------------------------------------- Jacobian */
static int bsr_pos(const oracle_solver* s, int row, int col) {
    int lo = s->rp[row], hi = s->rp[row + 1];
    while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (s->cols[mid] < col) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

/* compute_dt (solver.hpp:256-287) then JacobianKernel::apply
 * (jacobian_kernel.hpp:74-270): first-order Picard blocks from cell-centre
 * states, alpha on the diagonal.  With Spalart-Allmaras the blocks are 6x6:
 * the mean-flow 5x5 part as above, and the nu_tilde row/column carries only
 * the d/d(rho nu_tilde) entry (new math, the reference module has no
 * Jacobian): upwind convection m+/rho_L, m-/rho_R; thin-layer diffusion
 * +-coef A/|d|/rho; at boundary faces the ghost's dependence on the owner
 * (wall -1/rho_g, symmetry/outflow +1/rho_g, inflow 0); the destruction
 * derivative V 2 cw1 fw nu/d^2 on the diagonal.  Mean flow and turbulence
 * are not coupled in the Jacobian (Picard). */
static void jacobian(oracle_solver* s, double cfl) {
    const cfdg_mesh_host* m = &s->m;
    const int n = s->n, nt = s->nt, ni = s->ni, nf = s->nf, bs = s->nv, b2 = bs * bs;
    for (int c = 0; c < n; ++c) {
        const double l = fmax(s->lam[c], 1e-14);
        s->alpha[c] = l * (1.0 / cfl) + m->cell_volume[c] * 0.0;
    }
    memset(s->vals, 0, sizeof(double) * (size_t)b2 * (size_t)s->nnzb);
    const double is = 1.0 / SA_SIGMA;
    for (int f = 0; f < nf; ++f) {
        const int inner = f < ni;
        const int c0 = m->face_owner[f], c1 = inner ? m->face_neigh[f] : n + (f - ni);
        const double nx = m->face_normal_x[f], ny = m->face_normal_y[f], nz = m->face_normal_z[f], A = m->face_area[f];
        double qL[5], qR[5], UL[5], UR[5], F[5], smax, dFL[25], dFR[25], Jv[25];
        for (int v = 0; v < 5; ++v) {
            qL[v] = s->q[v * nt + c0];
            qR[v] = s->q[v * nt + c1];
        }
        prim2cons(s, qL, UL);
        prim2cons(s, qR, UR);
        hllc(s, UL, UR, nx, ny, nz, A, F, &smax);
        euler_jac(s, UL, nx, ny, nz, dFL);
        euler_jac(s, UR, nx, ny, nz, dFR);
        for (int i = 0; i < 25; ++i) {
            dFL[i] *= 0.5 * A;
            dFR[i] *= 0.5 * A;
        }
        for (int i = 0; i < 5; ++i) {
            dFL[i * 6] += 0.5 * smax * A;
            dFR[i * 6] -= 0.5 * smax * A;
        }
        if (s->visc) {
            const double mutL = s->sa ? s->mut[c0] : 0.0;
            const double mutR = (s->sa && inner) ? s->mut[c1] : 0.0;
            const int full = s->cfg.jacobian == CFDG_JAC_THIN_LAYER;
            double wv = 1.0, wt = 1.0;
            if (full && !inner) {
                const int kind = s->bcp[m->face_patch[f]].kind;
                if (kind == CFDG_BC_NO_SLIP_WALL || kind == CFDG_BC_NO_SLIP_WALL_HEAT_FLUX) wv = 2.0;
                if (kind == CFDG_BC_NO_SLIP_WALL) wt = 2.0;
            }
            viscous_jac(s, f, qL, qR, mutL, mutR, A, Jv, full, wv, wt);
            for (int i = 0; i < 25; ++i) {
                dFL[i] += Jv[i];
                dFR[i] += -Jv[i];
            }
        }
        double sL = 0.0, sR = 0.0; /* d F_nu / d (rho nu_tilde) of the two sides */
        if (s->sa) {
            const double mf = s->mdot[f], id = s->finv_d[f];
            if (inner) {
                const double Tf = 0.5 * (qL[4] + qR[4]);
                const double rho_f = 0.5 * (s->rho[c0] + s->rho[c1]);
                const double nu_f = 0.5 * (s->nu[c0] + s->nu[c1]);
                const double cd = is * (sutherland(Tf) + rho_f * nu_f) * A * id;
                sL = (fmax(mf, 0.0) + cd) / s->rho[c0];
                sR = (fmin(mf, 0.0) - cd) / s->rho[c1];
            } else {
                const int b = f - ni;
                const bcp_t* P = &s->bcp[m->face_patch[f]];
                const double rho_g = qR[0] / (s->R * qR[4]);
                const int inflow = (P->sa_kind == 1 || P->sa_kind == 2) && mf < 0.0;
                const double nu_g = inflow ? s->nu_inf : s->rhonu_g[b] / rho_g;
                const double Tf = 0.5 * (qL[4] + qR[4]);
                const double rho_f = 0.5 * (s->rho[c0] + rho_g);
                const double cd = is * (sutherland(Tf) + rho_f * 0.5 * (s->nu[c0] + nu_g)) * A * id;
                double dg = 0.0; /* d nu_g / d (rho nu_tilde)_owner */
                if (!inflow) dg = (P->sa_kind == 0) ? -1.0 / rho_g : (P->sa_kind == 1 ? 0.0 : 1.0 / rho_g);
                sL = (inflow ? 0.0 : mf / s->rho[c0]) + cd * (1.0 / s->rho[c0] - dg);
            }
        }
        double* a00 = s->vals + (size_t)b2 * s->diag[c0];
        if (inner) {
            double* a01 = s->vals + (size_t)b2 * bsr_pos(s, c0, c1);
            double* a11 = s->vals + (size_t)b2 * s->diag[c1];
            double* a10 = s->vals + (size_t)b2 * bsr_pos(s, c1, c0);
            for (int r = 0; r < 5; ++r)
                for (int k = 0; k < 5; ++k) {
                    a00[r * bs + k] += dFL[r * 5 + k];
                    a01[r * bs + k] += dFR[r * 5 + k];
                }
            for (int r = 0; r < 5; ++r)
                for (int k = 0; k < 5; ++k) {
                    a11[r * bs + k] -= dFR[r * 5 + k];
                    a10[r * bs + k] -= dFL[r * 5 + k];
                }
            if (s->sa) {
                a00[35] += sL;
                a01[35] += sR;
                a11[35] -= sR;
                a10[35] -= sL;
            }
        } else {
            for (int r = 0; r < 5; ++r)
                for (int k = 0; k < 5; ++k) a00[r * bs + k] += dFL[r * 5 + k];
            if (s->sa) a00[35] += sL;
        }
    }
    for (int c = 0; c < n; ++c) {
        double* d = s->vals + (size_t)b2 * s->diag[c];
        for (int i = 0; i < 5; ++i) d[i * (bs + 1)] += s->alpha[c];
        if (s->sa) {
            const double rho = s->rho[c], nu = s->nu[c];
            const double dd = fmax(s->dist[c], SA_MIN_WALL_DIST);
            const double fw = sa_fw(s, c);
            const double id2 = 1.0 / (dd * dd);
            d[35] += m->cell_volume[c] * 2.0 * SA_CW1 * fw * nu * id2 + s->alpha[c];
            (void)rho;
        }
    }
}

void oracle_jacobian(oracle_solver* s, double cfl, double* alpha, double* values) {
    jacobian(s, cfl);
    if (alpha) memcpy(alpha, s->alpha, sizeof(double) * (size_t)s->n);
    if (values) memcpy(values, s->vals, sizeof(double) * (size_t)s->nv * s->nv * (size_t)s->nnzb);
}

/* ----------------------------------------------------------- linear algebra */
/* bsr_spmv<BS> (linalg/bsr_helpers.hpp:138-203). */
void oracle_bsr_spmv(int n, int bs, const int32_t* rp, const int32_t* cols, const double* vals, const double* x,
                     double* y, double alpha, double beta) {
    const int b2 = bs * bs;
    if (alpha == 0.0) {
        for (size_t i = 0; i < (size_t)n * bs; ++i) y[i] = (beta == 0.0) ? 0.0 : y[i] * beta;
        return;
    }
    double acc[8];
    for (int i = 0; i < n; ++i) {
        for (int ii = 0; ii < bs; ++ii) acc[ii] = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const double* a = vals + (size_t)k * b2;
            const double* xb = x + (size_t)cols[k] * bs;
            for (int ii = 0; ii < bs; ++ii) {
                double t = 0.0;
                for (int jj = 0; jj < bs; ++jj) t += a[ii * bs + jj] * xb[jj];
                acc[ii] += t;
            }
        }
        double* yb = y + (size_t)i * bs;
        for (int ii = 0; ii < bs; ++ii) {
            if (alpha == 1.0 && beta == 0.0) yb[ii] = acc[ii];
            else if (beta == 1.0) yb[ii] += alpha * acc[ii];
            else if (beta == 0.0) yb[ii] = alpha * acc[ii];
            else yb[ii] = alpha * acc[ii] + beta * yb[ii];
        }
    }
}

/* lu_factor_block / lu_solve_block (linalg/bsr_helpers.hpp:278-353). */
static int lu_factor(double* a, int bs, int* piv) {
    for (int k = 0; k < bs; ++k) {
        int m = k;
        double mx = fabs(a[k * bs + k]);
        for (int i = k + 1; i < bs; ++i)
            if (fabs(a[i * bs + k]) > mx) {
                mx = fabs(a[i * bs + k]);
                m = i;
            }
        piv[k] = m;
        if (mx == 0.0) return 0;
        if (m != k)
            for (int j = 0; j < bs; ++j) {
                const double t = a[k * bs + j];
                a[k * bs + j] = a[m * bs + j];
                a[m * bs + j] = t;
            }
        const double id = 1.0 / a[k * bs + k];
        for (int i = k + 1; i < bs; ++i) {
            const double l = a[i * bs + k] * id;
            a[i * bs + k] = l;
            for (int j = k + 1; j < bs; ++j) a[i * bs + j] -= l * a[k * bs + j];
        }
    }
    return 1;
}

static void lu_solve(const double* lu, const int* piv, int bs, double* b) {
    for (int k = 0; k < bs; ++k)
        if (piv[k] != k) {
            const double t = b[k];
            b[k] = b[piv[k]];
            b[piv[k]] = t;
        }
    for (int i = 1; i < bs; ++i) {
        double s = b[i];
        for (int j = 0; j < i; ++j) s -= lu[i * bs + j] * b[j];
        b[i] = s;
    }
    for (int i = bs - 1; i >= 0; --i) {
        double s = b[i];
        for (int j = i + 1; j < bs; ++j) s -= lu[i * bs + j] * b[j];
        b[i] = s / lu[i * bs + i];
    }
}

typedef struct {
    int n, bs;
    const int32_t *rp, *cols;
    const double* vals;
    int32_t* diag;
    double* lu;
    int* piv;
    int sweeps;
} sgs_t;

/* SgsPreconditioner::setup, BSR branch (src/linalg/preconditioners.cpp:62-93). */
static int sgs_setup(sgs_t* P, int n, int bs, const int32_t* rp, const int32_t* cols, const double* vals, int sweeps) {
    P->n = n;
    P->bs = bs;
    P->rp = rp;
    P->cols = cols;
    P->vals = vals;
    P->sweeps = sweeps;
    P->diag = (int32_t*)xcalloc((size_t)n, 4);
    P->lu = (double*)xcalloc((size_t)n * bs * bs, 8);
    P->piv = (int*)xcalloc((size_t)n * bs, sizeof(int));
    for (int i = 0; i < n; ++i) {
        P->diag[i] = -1;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            if (cols[k] == i) P->diag[i] = k;
        if (P->diag[i] < 0) return 0;
        memcpy(P->lu + (size_t)i * bs * bs, vals + (size_t)P->diag[i] * bs * bs, sizeof(double) * bs * bs);
        if (!lu_factor(P->lu + (size_t)i * bs * bs, bs, P->piv + (size_t)i * bs)) return 0;
    }
    return 1;
}

static void sgs_free(sgs_t* P) {
    free(P->diag);
    free(P->lu);
    free(P->piv);
}

/* bsr_sgs_sweep<BS> (bsr_helpers.hpp:389-435), SgsPreconditioner::apply
 * (preconditioners.cpp:171-194): z = 0, forward then backward sweep. */
static void sgs_apply(const sgs_t* P, const double* r, double* z) {
    const int n = P->n, bs = P->bs, b2 = bs * bs;
    memset(z, 0, sizeof(double) * (size_t)n * bs);
    double s[8];
    for (int sw = 0; sw < P->sweeps; ++sw)
        for (int dir = 0; dir < 2; ++dir)
            for (int cnt = 0; cnt < n; ++cnt) {
                const int i = dir == 0 ? cnt : n - 1 - cnt;
                for (int ii = 0; ii < bs; ++ii) s[ii] = r[(size_t)i * bs + ii];
                for (int k = P->rp[i]; k < P->rp[i + 1]; ++k) {
                    if (k == P->diag[i]) continue;
                    const double* a = P->vals + (size_t)k * b2;
                    const double* zb = z + (size_t)P->cols[k] * bs;
                    for (int ii = 0; ii < bs; ++ii) {
                        double t = 0.0;
                        for (int jj = 0; jj < bs; ++jj) t += a[ii * bs + jj] * zb[jj];
                        s[ii] -= t;
                    }
                }
                lu_solve(P->lu + (size_t)i * b2, P->piv + (size_t)i * bs, bs, s);
                for (int ii = 0; ii < bs; ++ii) z[(size_t)i * bs + ii] = s[ii];
            }
}

int oracle_sgs_apply(int n, int bs, const int32_t* rp, const int32_t* cols, const double* vals, const double* r,
                     double* z, int sweeps) {
    sgs_t P;
    const int ok = sgs_setup(&P, n, bs, rp, cols, vals, sweeps);
    if (ok) sgs_apply(&P, r, z);
    sgs_free(&P);
    return ok ? 0 : -1;
}

static double dot(const double* a, const double* b, size_t N) {
    double s = 0.0;
    for (size_t i = 0; i < N; ++i) s += a[i] * b[i];
    return s;
}

/* BiCGSTAB::solve (src/linalg/bicgstab.cpp:42-201), right-preconditioned,
 * five fused inner products, true-norm refresh every 32 iterations.
 * status: 0 converged, 1 diverged, 2 max iterations. */
static int bicgstab_core(int n, int bs, const int32_t* rp, const int32_t* cols, const double* vals,
                         const sgs_t* M, double rtol, double atol, int max_it, double* x, const double* b,
                         int* iters, int* status, double* r_init, double* r_final) {
    const size_t N = (size_t)n * bs;
    double* w = (double*)xcalloc(8 * N, 8);
    double *r = w, *r0 = w + N, *p = w + 2 * N, *v = w + 3 * N, *sv = w + 4 * N, *t = w + 5 * N, *ph = w + 6 * N,
           *sh = w + 7 * N;
    oracle_bsr_spmv(n, bs, rp, cols, vals, x, v, 1.0, 0.0);
    for (size_t i = 0; i < N; ++i) r[i] = b[i] + (-1.0) * v[i];
    const double bnorm = sqrt(dot(b, b, N));
    double rnorm = sqrt(dot(r, r, N));
    const double scale = bnorm > 0.0 ? bnorm : 1.0;
    const double tol = fmax(atol, rtol * scale);
    *r_init = rnorm;
    int st = 2, it = 0;
    if (!isfinite(rnorm)) st = 1;
    else if (rnorm <= tol) st = 0;
    if (st == 2) {
        memcpy(r0, r, sizeof(double) * N);
        double rho = rnorm * rnorm, rho_old = 1.0, alpha = 1.0, omega = 1.0;
        for (;;) {
            if (it >= max_it) {
                st = 2;
                break;
            }
            ++it;
            if (it == 1) {
                memcpy(p, r, sizeof(double) * N);
            } else {
                const double beta = (rho / rho_old) * (alpha / omega);
                if (!isfinite(beta)) {
                    st = 1;
                    break;
                }
                for (size_t i = 0; i < N; ++i) {
                    double pv = beta * p[i];
                    pv = pv + (-beta * omega) * v[i];
                    p[i] = pv + 1.0 * r[i];
                }
            }
            if (M) sgs_apply(M, p, ph);
            else memcpy(ph, p, sizeof(double) * N);
            oracle_bsr_spmv(n, bs, rp, cols, vals, ph, v, 1.0, 0.0);
            const double gamma = dot(r0, v, N);
            if (!isfinite(gamma) || gamma == 0.0) {
                st = 1;
                break;
            }
            alpha = rho / gamma;
            for (size_t i = 0; i < N; ++i) sv[i] = r[i] + (-alpha) * v[i];
            if (M) sgs_apply(M, sv, sh);
            else memcpy(sh, sv, sizeof(double) * N);
            oracle_bsr_spmv(n, bs, rp, cols, vals, sh, t, 1.0, 0.0);
            const double tt = dot(t, t, N), ts = dot(t, sv, N), r0t = dot(r0, t, N), r0s = dot(r0, sv, N),
                         ss = dot(sv, sv, N);
            if (!isfinite(ts) || !isfinite(tt) || tt == 0.0) {
                st = 1;
                break;
            }
            const double om = ts / tt;
            for (size_t i = 0; i < N; ++i) {
                double xv = x[i] + alpha * ph[i];
                x[i] = xv + om * sh[i];
                r[i] = sv[i] + (-om) * t[i];
            }
            rnorm = sqrt(fmax(ss - 2.0 * om * ts + om * om * tt, 0.0));
            const double rho_new = r0s - om * r0t;
            if (!isfinite(rnorm) || !isfinite(om) || om == 0.0) {
                st = 1;
                break;
            }
            if (it % 32 == 0) rnorm = sqrt(dot(r, r, N));
            if (rnorm <= tol) {
                st = 0;
                break;
            }
            if (!isfinite(rho_new) || rho_new == 0.0) {
                st = 1;
                break;
            }
            rho_old = rho;
            rho = rho_new;
            omega = om;
        }
    }
    *iters = it;
    *status = st;
    *r_final = rnorm;
    free(w);
    return 0;
}

int oracle_bicgstab(int n, int bs, const int32_t* rp, const int32_t* cols, const double* vals, int precond,
                    double rtol, double atol, int max_it, double* x, const double* b, int* iterations, int* status,
                    double* r_init, double* r_final) {
    sgs_t P;
    int use = 0;
    if (precond == CFDG_PC_SGS) {
        if (!sgs_setup(&P, n, bs, rp, cols, vals, 1)) {
            sgs_free(&P);
            return -1;
        }
        use = 1;
    }
    bicgstab_core(n, bs, rp, cols, vals, use ? &P : NULL, rtol, atol, max_it, x, b, iterations, status, r_init,
                  r_final);
    if (use) sgs_free(&P);
    return 0;
}

/* ---------------------------------------------------------------- Newton */
/* BackwardEuler::advance (time/implicit_euler.hpp:34-92); with
 * Spalart-Allmaras the sixth variable is updated in the same solve and
 * clamped at zero (SpalartAllmaras::post_stage, spalart_allmaras.hpp:435-441). */
int oracle_newton_step(oracle_solver* s, double cfl, double* l2, int* krylov) {
    const int n = s->n, bs = s->nv;
    residual(s);
    jacobian(s, cfl);
    const size_t N = (size_t)n * bs;
    double* b = (double*)xcalloc(N, 8);
    double* du = (double*)xcalloc(N, 8);
    for (int c = 0; c < n; ++c)
        for (int v = 0; v < bs; ++v) b[(size_t)c * bs + v] = -s->res[(size_t)v * n + c];
    int it = 0, st = 2;
    double r0, rf;
    const cfdg_config* cfg = &s->cfg;
    if (cfg->precond == CFDG_PC_SGS) {
        sgs_t P;
        if (!sgs_setup(&P, n, bs, s->rp, s->cols, s->vals, cfg->sgs_sweeps > 0 ? cfg->sgs_sweeps : 1)) {
            sgs_free(&P);
            free(b);
            free(du);
            return -1;
        }
        bicgstab_core(n, bs, s->rp, s->cols, s->vals, &P, cfg->lin_rel_tol, cfg->lin_abs_tol,
                      cfg->lin_max_iterations, du, b, &it, &st, &r0, &rf);
        sgs_free(&P);
    } else {
        bicgstab_core(n, bs, s->rp, s->cols, s->vals, NULL, cfg->lin_rel_tol, cfg->lin_abs_tol,
                      cfg->lin_max_iterations, du, b, &it, &st, &r0, &rf);
    }
    for (int v = 0; v < bs; ++v)
        for (int c = 0; c < n; ++c) {
            double x = s->U[(size_t)v * n + c] + du[(size_t)c * bs + v];
            if (v == 5 && x < 0.0) x = 0.0;
            s->U[(size_t)v * n + c] = x;
        }
    /* residual_norms (solver.hpp:740-756) of the evaluated R(U) */
    for (int v = 0; v < bs; ++v) {
        double acc = 0.0;
        for (int c = 0; c < n; ++c) acc += s->res[(size_t)v * n + c] * s->res[(size_t)v * n + c];
        l2[v] = sqrt(acc / (double)(n > 0 ? n : 1));
    }
    if (krylov) {
        krylov[0] = it;
        krylov[1] = st;
    }
    free(b);
    free(du);
    return 0;
}

/* Keep (1) or recompute (0) the MUSCL limiter values at later evaluations:
 * the library's cfdg_solver_freeze_limiter, which the reference lacks. */
void oracle_freeze_limiter(oracle_solver* s, int frozen) { s->phi_frozen = frozen ? 1 : 0; }

void oracle_sa_fields(const oracle_solver* s, double* dist, double* nu, double* mut, double* gnu) {
    if (!s->sa) return;
    const size_t n = (size_t)s->n, nt = (size_t)s->nt;
    if (dist) memcpy(dist, s->dist, sizeof(double) * n);
    if (nu) memcpy(nu, s->nu, sizeof(double) * n);
    if (mut) memcpy(mut, s->mut, sizeof(double) * nt);
    if (gnu) memcpy(gnu, s->gnu, sizeof(double) * 3 * nt);
}
