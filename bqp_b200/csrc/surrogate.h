// Learned gravity surrogate (surrogate.cu): model state and entry points.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>

namespace bqp {
namespace sg {

constexpr int kH = 256;  // hidden width
// FP32 parameter vector: W0[256][4] b0[256] W1..W3[256][256] b1..b3[256] W4[3][256] b4[3]
constexpr int kOffW0 = 0;
constexpr int kOffB0 = kOffW0 + kH * 4;
constexpr int kOffW1 = kOffB0 + kH;
constexpr int kOffB1 = kOffW1 + 3 * kH * kH;
constexpr int kOffW4 = kOffB1 + 3 * kH;
constexpr int kOffB4 = kOffW4 + 3 * kH;
constexpr int kParams = kOffB4 + 3;

struct Scale {
    double R;       // reference radius of the output scaling (km)
    double r_mid;   // radius input: (r - r_mid) / r_half
    double r_half;
};

}  // namespace sg

struct TrainArgs {
    int64_t samples;
    int32_t epochs;
    int32_t batch;  // multiple of 128
    double lr;
    uint64_t seed;
};

// fills acc[n][3] with an exact field at pos[n][3] (device buffers)
using FieldFn = std::function<cudaError_t(int64_t, const double*, double*)>;

struct Model {
    sg::Scale scale{6378.13646, 7078.0, 500.0};
    double sigma = 1.0;
    int64_t samples = 0;
    int batch_cap = 0;
    bool trained = false;
    float *P = nullptr, *G = nullptr, *m1 = nullptr, *m2 = nullptr;
    __nv_bfloat16 *W = nullptr, *Wt = nullptr;
    __nv_bfloat16* Wtile = nullptr;  // the hidden matrices in the tensor cores' shared-memory layout
    float *x = nullptr, *t = nullptr;  // training set
    float *xb = nullptr, *tb = nullptr;
    float* z[4] = {nullptr, nullptr, nullptr, nullptr};
    __nv_bfloat16* h[4] = {nullptr, nullptr, nullptr, nullptr};
    __nv_bfloat16* dz[4] = {nullptr, nullptr, nullptr, nullptr};
    __nv_bfloat16 *dzt = nullptr, *ht = nullptr;
    float *dh = nullptr, *y = nullptr, *dy = nullptr;
    double* dsum = nullptr;
    int* derr = nullptr;  // [0] GEMM wait timeout, then sigma (double at +8), loss sum (double at +16)

    ~Model();
    void release();
    cudaError_t alloc_params();
    cudaError_t alloc_batch(int B);
};

cudaError_t train(Model& M, const TrainArgs& a, const FieldFn& full, const FieldFn& low, cudaStream_t st,
                  double* loss_per_epoch);
cudaError_t infer(Model& M, int64_t n, const double* pos, double* acc, int add, cudaStream_t st);
// the same through one fused kernel (weights staged per layer, activations
// kept on chip); adds the residual to acc
cudaError_t infer_fused(Model& M, int64_t n, const double* pos, double* acc, int* err, cudaStream_t st);
cudaError_t forward_backward(Model& M, int B, bool train, cudaStream_t st);
cudaError_t refresh_bf16(Model& M, cudaStream_t st);
cudaError_t upload_params(Model& M, const float* host, cudaStream_t st);

}  // namespace bqp
