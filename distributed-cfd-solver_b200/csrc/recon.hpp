// Gradient and limiter operators on caller-owned device arrays: the GPU
// counterparts of GradientOperator::apply_set
// (include/cfd/numerics/gradient/gradient_operator.hpp:16-44) and
// Muscl<L>::compute_limiters (include/cfd/numerics/reconstruction/muscl.hpp:25-105)
// for callers that keep their own fields (cfdg_recon_* in cfdg.h).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "cfdg.h"
#include "solver.hpp"

namespace cfdg {

// Up to kMaxVars scalar fields per launch, passed by value.
struct ReconPtrs {
    const double* q[kMaxVars];
    const double* gx[kMaxVars];
    const double* gy[kMaxVars];
    const double* gz[kMaxVars];
    double* out[3 * kMaxVars];  // gradient: gx, gy, gz planes per variable; limiter: phi per variable
};

template <int NV>
void launch_gradient_ptrs(const DevMesh& m, const ReconPtrs& p, cudaStream_t s);
template <int NV>
void launch_limiter_ptrs(const DevMesh& m, const ReconPtrs& p, int limiter, double k3, cudaStream_t s);

class ReconOperator {
public:
    ReconOperator(int device, const cfdg_mesh_host& mesh, int gradient, int limiter, double venkat_k);
    int device() const { return device_; }
    int32_t n_cells() const { return dm_.n; }
    // grad(q_v) on the cells for v < nvars
    void gradient(const double* const* q, double* const* gx, double* const* gy, double* const* gz, int nvars,
                  cudaStream_t s);
    // phi_v from q_v and its gradient for v < nvars
    void limiter(const double* const* q, const double* const* gx, const double* const* gy, const double* const* gz,
                 double* const* phi, int nvars, cudaStream_t s);

private:
    int device_;
    int limiter_;
    double k3_;
    DevMesh dm_{};
    DevArray<int32_t> c2f_off_, c2f_, c2c_off_, c2c_, g_col_;
    DevArray<int64_t> g_soff_;
    DevArray<double> fcx_, fcy_, fcz_, ccx_, ccy_, ccz_, vol_, g_wx_, g_wy_, g_wz_;
};

}  // namespace cfdg
