// Host side of the learned Newton initial guess (network + dataset).
#include "guess.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>

#include "solver.hpp"

namespace cfdg {

namespace {

template <typename T>
T* dev_alloc(std::size_t n, const char* what) {
    T* p = nullptr;
    if (cudaMalloc(reinterpret_cast<void**>(&p), std::max<std::size_t>(n, 1) * sizeof(T)) != cudaSuccess)
        throw Failure{CFDG_ERR_NOMEM, std::string("out of device memory: ") + what};
    return p;
}

uint16_t to_bf16(float x) {  // round to nearest even (finite inputs)
    uint32_t u;
    std::memcpy(&u, &x, 4);
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7FFFu + lsb;
    return static_cast<uint16_t>(u >> 16);
}

}  // namespace

Mlp::Mlp(int device, int nvars, uint64_t seed) : device_(device), nvars_(nvars) {
    if (nvars < 1 || nvars > kMlpOut || 8 * nvars > kMlpIn)
        throw Failure{CFDG_ERR_INVALID, "learned guess supports 1..6 variables"};
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    int sms = 1;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "device attribute");
    grid_train_ = sms;      // one CTA per SM (512 tensor-memory columns each)
    grid_fwd_ = 4 * sms;    // 128 columns each
    params_ = dev_alloc<float>(kMlpParams, "mlp params");
    m_ = dev_alloc<float>(kMlpParams, "mlp adam m");
    v_ = dev_alloc<float>(kMlpParams, "mlp adam v");
    grad_ = dev_alloc<float>(kMlpParams, "mlp grad");
    loss_ = dev_alloc<float>(1, "mlp loss");
    partials_ = dev_alloc<float>(static_cast<std::size_t>(grid_train_) * (kMlpParams + 1), "mlp partials");
    w_ = dev_alloc<uint16_t>(kMlpHid * kMlpIn + kMlpHid * kMlpHid + kMlpOut * kMlpHid, "mlp bf16 weights");
    err_ = dev_alloc<int>(1, "mlp error flag");
    cuda_check(cudaMemset(m_, 0, kMlpParams * sizeof(float)), "memset");
    cuda_check(cudaMemset(v_, 0, kMlpParams * sizeof(float)), "memset");
    cuda_check(cudaMemset(err_, 0, sizeof(int)), "memset");
    // uniform(-a, a) with a = sqrt(6 / fan_in) (ReLU layers) and a small
    // output layer so that an untrained network predicts ~0
    std::vector<float> p(kMlpParams, 0.0f);
    std::mt19937_64 g(seed);
    std::uniform_real_distribution<double> u(-1.0, 1.0);
    const double a1 = std::sqrt(6.0 / kMlpIn), a2 = std::sqrt(6.0 / kMlpHid), a3 = 0.1 * std::sqrt(6.0 / kMlpHid);
    for (int i = 0; i < kMlpHid * kMlpIn; ++i) p[kOffW1 + i] = static_cast<float>(a1 * u(g));
    for (int i = 0; i < kMlpHid * kMlpHid; ++i) p[kOffW2 + i] = static_cast<float>(a2 * u(g));
    for (int i = 0; i < kMlpOut * kMlpHid; ++i) p[kOffW3 + i] = static_cast<float>(a3 * u(g));
    set_params(p.data());
}

Mlp::~Mlp() {
    for (void* q : {static_cast<void*>(params_), static_cast<void*>(m_), static_cast<void*>(v_),
                    static_cast<void*>(grad_), static_cast<void*>(loss_), static_cast<void*>(partials_),
                    static_cast<void*>(w_), static_cast<void*>(err_)})
        if (q) cudaFree(q);
}

MlpDev Mlp::dev() const {
    MlpDev d;
    d.w1 = w_;
    d.w2 = w_ + kMlpHid * kMlpIn;
    d.w3 = w_ + kMlpHid * kMlpIn + kMlpHid * kMlpHid;
    d.params = params_;
    d.nout = nvars_;
    return d;
}

void Mlp::set_params(const float* p) {
    std::vector<float> q(p, p + kMlpParams);
    // outputs beyond nvars carry no loss: keep their weights at zero
    for (int o = nvars_; o < kMlpOut; ++o) {
        for (int i = 0; i < kMlpHid; ++i) q[kOffW3 + o * kMlpHid + i] = 0.0f;
        q[kOffB3 + o] = 0.0f;
    }
    cuda_check(cudaMemcpy(params_, q.data(), kMlpParams * sizeof(float), cudaMemcpyHostToDevice), "H2D");
    std::vector<uint16_t> w(kMlpHid * kMlpIn + kMlpHid * kMlpHid + kMlpOut * kMlpHid);
    std::size_t k = 0;
    for (int i = 0; i < kMlpHid * kMlpIn; ++i) w[k++] = to_bf16(q[kOffW1 + i]);
    for (int i = 0; i < kMlpHid * kMlpHid; ++i) w[k++] = to_bf16(q[kOffW2 + i]);
    for (int i = 0; i < kMlpOut * kMlpHid; ++i) w[k++] = to_bf16(q[kOffW3 + i]);
    cuda_check(cudaMemcpy(w_, w.data(), w.size() * sizeof(uint16_t), cudaMemcpyHostToDevice), "H2D");
    step_ = 0;
    cuda_check(cudaMemset(m_, 0, kMlpParams * sizeof(float)), "memset");
    cuda_check(cudaMemset(v_, 0, kMlpParams * sizeof(float)), "memset");
}

void Mlp::get_params(float* p) {
    cuda_check(cudaMemcpy(p, params_, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost), "D2H");
}

void Mlp::check_err(cudaStream_t s) {
    int e = 0;
    cuda_check(cudaMemcpyAsync(&e, err_, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "mlp sync");
    if (e) {
        cudaMemsetAsync(err_, 0, sizeof(int), s);
        throw Failure{CFDG_ERR_CUDA, "tensor-core MLP kernel: wait on the MMA completion timed out"};
    }
}

void Mlp::forward(const uint16_t* feat, int64_t rows, const double* scale, double* out, cudaStream_t s) {
    launch_mlp_forward(dev(), feat, rows, scale, nvars_, out, err_, grid_fwd_, s);
    ++launches_;
    cuda_check(cudaGetLastError(), "mlp forward launch");
}

float Mlp::run_grad(const uint16_t* X, const float* T, int64_t rows, bool adam, float lr, cudaStream_t s) {
    if (rows <= 0) throw Failure{CFDG_ERR_INVALID, "empty batch"};
    launch_mlp_grad(dev(), X, T, rows, partials_, err_, grid_train_, s);
    if (adam) ++step_;
    const double inv = 1.0 / (double(rows) * nvars_);
    uint16_t* w1 = w_;
    uint16_t* w2 = w_ + kMlpHid * kMlpIn;
    uint16_t* w3 = w2 + kMlpHid * kMlpHid;
    launch_mlp_adam(params_, m_, v_, w1, w2, w3, partials_, grid_train_, inv, lr, 0.9f, 0.999f, 1e-8f,
                    std::max(step_, 1), adam, grad_, loss_, s);
    launches_ += adam ? 3 : 2;
    cuda_check(cudaGetLastError(), "mlp train launch");
    float loss = 0.0f;
    cuda_check(cudaMemcpyAsync(&loss, loss_, sizeof(float), cudaMemcpyDeviceToHost, s), "D2H");
    check_err(s);
    return loss;
}

float Mlp::gradient(const uint16_t* X, const float* T, int64_t rows, float* grad_host, cudaStream_t s) {
    const float loss = run_grad(X, T, rows, false, 0.0f, s);
    if (grad_host) {
        cuda_check(cudaMemcpyAsync(grad_host, grad_, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, s), "D2H");
        cuda_check(cudaStreamSynchronize(s), "sync");
    }
    return loss;
}

float Mlp::adam_step(const uint16_t* X, const float* T, int64_t rows, float lr, cudaStream_t s) {
    return run_grad(X, T, rows, true, lr, s);
}

float Mlp::train(const Dataset& ds, int epochs, int batch, float lr, uint64_t seed, cudaStream_t s) {
    if (ds.nvars() != nvars_) throw Failure{CFDG_ERR_INVALID, "dataset and network variable counts differ"};
    const int64_t n = ds.size();
    if (n <= 0) throw Failure{CFDG_ERR_INVALID, "empty dataset"};
    batch = std::max(batch, kMlpTile);
    const int64_t nb = (n + batch - 1) / batch;
    std::vector<int64_t> order(static_cast<std::size_t>(nb));
    std::iota(order.begin(), order.end(), int64_t(0));
    std::mt19937_64 g(seed);
    float last = 0.0f;
    for (int e = 0; e < epochs; ++e) {
        std::shuffle(order.begin(), order.end(), g);
        double acc = 0.0;
        for (int64_t k : order) {
            const int64_t r0 = k * batch, rows = std::min<int64_t>(batch, n - r0);
            acc += double(adam_step(ds.X() + r0 * kMlpIn, ds.T() + r0 * kMlpOut, rows, lr, s)) * double(rows);
        }
        last = static_cast<float>(acc / double(n));
    }
    return last;
}

Dataset::Dataset(int device, int nvars, int64_t capacity) : device_(device), nvars_(nvars), capacity_(capacity) {
    if (capacity <= 0) throw Failure{CFDG_ERR_INVALID, "dataset capacity must be positive"};
    if (nvars < 1 || nvars > 6) throw Failure{CFDG_ERR_INVALID, "dataset supports 1..6 variables"};
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    X_ = dev_alloc<uint16_t>(static_cast<std::size_t>(capacity) * kMlpIn, "dataset features");
    T_ = dev_alloc<float>(static_cast<std::size_t>(capacity) * kMlpOut, "dataset targets");
}

Dataset::~Dataset() {
    if (X_) cudaFree(X_);
    if (T_) cudaFree(T_);
}

void Dataset::append_host(const uint16_t* X, const float* T, int64_t rows) {
    const int64_t r0 = size_;
    const int64_t g = reserve(rows);
    if (g < rows) throw Failure{CFDG_ERR_INVALID, "dataset capacity exceeded"};
    cuda_check(cudaMemcpy(X_ + r0 * kMlpIn, X, rows * kMlpIn * sizeof(uint16_t), cudaMemcpyHostToDevice), "H2D");
    cuda_check(cudaMemcpy(T_ + r0 * kMlpOut, T, rows * kMlpOut * sizeof(float), cudaMemcpyHostToDevice), "H2D");
}

void Dataset::read_host(uint16_t* X, float* T, int64_t rows) const {
    if (rows > size_) throw Failure{CFDG_ERR_INVALID, "reading past the dataset size"};
    if (X) cuda_check(cudaMemcpy(X, X_, rows * kMlpIn * sizeof(uint16_t), cudaMemcpyDeviceToHost), "D2H");
    if (T) cuda_check(cudaMemcpy(T, T_, rows * kMlpOut * sizeof(float), cudaMemcpyDeviceToHost), "D2H");
}

}  // namespace cfdg
