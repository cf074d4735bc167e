// Device-resident BiCGSTAB scalars and launcher declarations.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.hpp"

namespace cfdg {

enum : int { KS_RUNNING = 0, KS_CONVERGED = 1, KS_DIVERGED = 2, KS_MAXIT = 3 };

// Scalars of BiCGSTAB::solve (src/linalg/bicgstab.cpp:42-201) kept on the
// device so that an iteration needs no host round trip.  `state` is the
// first member: kernels early-exit when it is not KS_RUNNING.
struct KrylovScalars {
    int state;
    int it;
    int max_it;
    int guess;  // in: 1 when x holds an initial guess that may be rejected; out: 2 when rejected
    int body_runs;  // device loop: iterations the graph body has run (bounds the loop by max_it)
    double rel_tol, abs_tol;
    double bnorm, scale, tol, initial, rnorm;
    double rho, rho_old, rho_new, alpha, omega, omega_new, beta;
};

// Up to five (a, b) vector pairs; a null pointer stands for the SpMV output.
struct DotSpec {
    const double* a[5];
    const double* b[5];
    int n;
};

// Jacobian-free product y = (alpha - V diag) x + (R(U + eps x) + b) / eps
// from the perturbed residual `resp` (SoA, cell order), with the dots `ds`;
// returns the partial count.
int launch_jf_combine(const DevMesh& m, int nv, const double* alpha, double diag, const double* x, const double* b,
                      const double* resp, const double* scal, double* y, const DotSpec& ds, double* partials,
                      const int* active, cudaStream_t s);

// y = alpha A x + beta y on rows [row_begin, n), optional fused dots
template <typename MT>
void launch_spmv_ex(const BsrView& A, const MT* vals, const double* x, double* y, double alpha, double beta,
                    const DotSpec& ds, double* partials, const int* active, cudaStream_t s, int32_t row_begin = 0);
// Last backward pass of the split multicolour sweep (colour 0 = rows
// [0, n_rows), `dinv` the inverse diagonal blocks) fused with y = A z and the
// dots on those rows; partials: sgs_last_spmv_blocks(n_rows, bs) * ds.n.
template <typename MT>
void launch_sgs_last_spmv(const BsrView& A, const MT* vals, const MT* dinv, int32_t n_rows, double* z, double* y,
                          const DotSpec& ds, double* partials, const int* active, cudaStream_t s);
int sgs_last_spmv_blocks(int32_t n_rows, int32_t bs);
// rows: the pass's row list, or null for the contiguous rows row0 ..
// inverse: `lu` holds D^-1 (launch_lu_setup with inverse)
template <typename MT>
void launch_sgs_rows_ex(const BsrView& A, const MT* vals, const MT* lu, const int8_t* piv, const int32_t* rows,
                        int32_t row0, int32_t n_rows, const double* r, double* z, int mode, bool inverse,
                        const int* active, cudaStream_t s);
// The whole level-scheduled symmetric sweep (forward levels, then backward
// levels; z zeroed by the caller) as one cooperative launch with a grid
// barrier per level; rows as (row, row_ptr[row], row_ptr[row+1], diag[row])
// records in level order.  False when the device or block size has no
// cooperative launch (the caller then launches level by level).
template <typename MT>
bool launch_sgs_level_coop(const BsrView& A, const MT* vals, const MT* lu, const int8_t* piv, const int4* fwd_rows,
                           const int32_t* fwd_off, int n_fwd, const int4* bwd_rows, const int32_t* bwd_off,
                           int n_bwd, const double* r, double* z, const int* active, cudaStream_t s);
void launch_krylov_init(int64_t len, const double* b, const double* v, double* r, double* r0, double* p,
                        double* partials, KrylovScalars* ks, cudaStream_t s);
// After launch_krylov_init: a rejected initial guess (||b - A x0|| >=
// ||b||) restarts from x = 0 (r = r0 = p = b).
void launch_krylov_guess_reset(int64_t len, const KrylovScalars* ks, const double* b, double* x, double* r, double* r0,
                               double* p, cudaStream_t s);
void launch_krylov_begin(KrylovScalars* ks, cudaStream_t s);
void launch_krylov_gamma(KrylovScalars* ks, const double* partials, int nblocks, cudaStream_t s);
void launch_krylov_s(int64_t len, const KrylovScalars* ks, const double* r, const double* v, double* sv,
                     cudaStream_t s);
void launch_krylov_omega(KrylovScalars* ks, const double* partials, int nblocks, cudaStream_t s);
void launch_krylov_update(int64_t len, const KrylovScalars* ks, double* x, const double* phat, const double* shat,
                          const double* sv, const double* tv, double* r, double* p, const double* v,
                          double* partials, cudaStream_t s);
void launch_krylov_post(KrylovScalars* ks, const double* partials, int nblocks, cudaStream_t s);
// Last node of the device loop's body: counts the body run and sets the
// while-condition to (state == running and runs < max_it).
void launch_krylov_cond(KrylovScalars* ks, cudaGraphConditionalHandle h, cudaStream_t s);

}  // namespace cfdg
