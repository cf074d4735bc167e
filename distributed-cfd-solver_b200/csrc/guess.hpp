// Host side of the learned Newton initial guess: the network (fp32 master
// weights, bf16 copies for the tensor cores, Adam state) and the device
// dataset of (features, dU) samples the solver writes out.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "device_common.cuh"
#include "mlp.hpp"

namespace cfdg {

int guess_sum_blocks(int32_t n);
void launch_guess_scales(int32_t n, const int32_t* row_of, int nv, const double* b, const double* dt,
                         const double* vol, const double* du_prev, double* partials, double* gscale, cudaStream_t s);
void launch_guess_features(const DevMesh& m, int nv, const double* U, const double* b, const double* dt,
                           const double* du_prev, const double* gscale, double cfl, uint16_t* feat, cudaStream_t s);
void launch_guess_append(int32_t n, const int32_t* row_of, int nv, int32_t stride, int32_t phase, int64_t count,
                         const uint16_t* feat, const double* du, const double* gscale, uint16_t* X, float* T,
                         cudaStream_t s);

class Dataset;

class Mlp {
public:
    Mlp(int device, int nvars, uint64_t seed);
    ~Mlp();
    int device() const { return device_; }
    int nvars() const { return nvars_; }
    MlpDev dev() const;
    void set_params(const float* p);  // host, kMlpParams values
    void get_params(float* p);
    // out[r * nv + v] = scale[v] * y_v (device arrays; stream ordered)
    void forward(const uint16_t* feat, int64_t rows, const double* scale, double* out, cudaStream_t s);
    // loss (mean squared error over rows x nvars) and, when grad_host is
    // set, its gradient; no update
    float gradient(const uint16_t* X, const float* T, int64_t rows, float* grad_host, cudaStream_t s);
    // one Adam step on the batch; returns the batch loss before the step
    float adam_step(const uint16_t* X, const float* T, int64_t rows, float lr, cudaStream_t s);
    // epochs over the dataset in shuffled contiguous batches; mean loss of the last epoch
    float train(const Dataset& ds, int epochs, int batch, float lr, uint64_t seed, cudaStream_t s);
    int64_t launches() const { return launches_; }

private:
    int device_, nvars_;
    float* params_ = nullptr;  // device fp32 master
    float* m_ = nullptr;
    float* v_ = nullptr;
    float* grad_ = nullptr;
    float* loss_ = nullptr;
    float* partials_ = nullptr;
    uint16_t* w_ = nullptr;  // bf16 W1 | W2 | W3
    int* err_ = nullptr;
    int grid_train_ = 1, grid_fwd_ = 1;
    int step_ = 0;
    int64_t launches_ = 0;
    float run_grad(const uint16_t* X, const float* T, int64_t rows, bool adam, float lr, cudaStream_t s);
    void check_err(cudaStream_t s);
};

class Dataset {
public:
    Dataset(int device, int nvars, int64_t capacity);
    ~Dataset();
    int device() const { return device_; }
    int nvars() const { return nvars_; }
    int64_t capacity() const { return capacity_; }
    int64_t size() const { return size_; }
    uint16_t* X() const { return X_; }
    float* T() const { return T_; }
    // reserves up to `count` rows at the end; returns the rows granted
    int64_t reserve(int64_t count) {
        const int64_t g = count < capacity_ - size_ ? count : capacity_ - size_;
        size_ += g > 0 ? g : 0;
        return g > 0 ? g : 0;
    }
    void append_host(const uint16_t* X, const float* T, int64_t rows);
    void read_host(uint16_t* X, float* T, int64_t rows) const;
    void clear() { size_ = 0; }

private:
    int device_, nvars_;
    int64_t capacity_, size_ = 0;
    uint16_t* X_ = nullptr;
    float* T_ = nullptr;
};

}  // namespace cfdg
