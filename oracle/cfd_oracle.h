/*
 * CPU restatement (plain C) of the reference solver's hot path, used as an
 * independent checker of the GPU library.  TEST INFRASTRUCTURE ONLY: the
 * tests, __graft_entry__.smoke() and bench.py's CPU baseline leg call it;
 * the product library never links it.
 *
 * Parity is pinned: tests/test_oracle_cpu.py checks every stage of this
 * restatement against the reference's own code (oracle/_ref, built from the
 * reference sources) and against the committed golden vectors.
 */
#ifndef CFD_ORACLE_H
#define CFD_ORACLE_H

#include <stdint.h>

#include "../include/cfdg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_solver oracle_solver;

/* kind 0 cell->faces, 1 cell->cells by face, 2 cell->cells by node; returns
 * the entry count, fills off (n+1) and val when val is non-null. */
int64_t oracle_connectivity(const cfdg_mesh_host* m, int kind, int32_t* off, int32_t* val);

int oracle_create(const cfdg_mesh_host* m, const cfdg_config* cfg, const cfdg_bc_desc* bcs, int nbc,
                  oracle_solver** out);
void oracle_destroy(oracle_solver* s);
int64_t oracle_nnzb(const oracle_solver* s);
int oracle_structure(const oracle_solver* s, int32_t* row_ptr, int32_t* cols);
void oracle_set_state(oracle_solver* s, const double* U, int64_t ld);
void oracle_get_state(const oracle_solver* s, double* U, int64_t ld);
/* residual pipeline: q (nv_q x nt), grad (nv x 3 x nt), phi (5 x n), res (nv x n), lam (n) */
void oracle_stages(oracle_solver* s, double* q, double* grad, double* phi, double* res, double* lam);
void oracle_jacobian(oracle_solver* s, double cfl, double* alpha, double* values);
/* one backward-Euler Newton step; l2 of R(U) before the update (nv values);
 * krylov[0]=iterations, krylov[1]=status; returns 0 */
int oracle_newton_step(oracle_solver* s, double cfl, double* l2, int* krylov);
int oracle_nvars(const oracle_solver* s);
/* Spalart-Allmaras fields: wall distance (n), nu_tilde (n), eddy viscosity
 * (n_total), nu_tilde gradient (3 x n_total); no-op without the model. */
void oracle_sa_fields(const oracle_solver* s, double* dist, double* nu, double* mut, double* gnu);
void oracle_freeze_limiter(oracle_solver* s, int frozen);

/* linear algebra on raw BSR arrays */
void oracle_bsr_spmv(int n, int bs, const int32_t* rp, const int32_t* cols, const double* vals, const double* x,
                     double* y, double alpha, double beta);
int oracle_sgs_apply(int n, int bs, const int32_t* rp, const int32_t* cols, const double* vals, const double* r,
                     double* z, int sweeps);
int oracle_bicgstab(int n, int bs, const int32_t* rp, const int32_t* cols, const double* vals, int precond,
                    double rtol, double atol, int max_it, double* x, const double* b, int* iterations, int* status,
                    double* r_init, double* r_final);

#ifdef __cplusplus
}
#endif
#endif
