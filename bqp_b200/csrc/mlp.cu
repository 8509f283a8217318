// The gravity surrogate's tensor-core building blocks: the BF16 GEMM of
// tc_gemm.cuh behind a launcher (C = A B^T, FP32 out).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "launch.h"
#include "tc_gemm.cuh"

namespace bqp {

__global__ void __launch_bounds__(tc::kThreads, 1)
    k_gemm_bf16(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B, float* __restrict__ C,
                int N, int K, int* err) {
    const int m0 = blockIdx.x * tc::kBM, n0 = blockIdx.y * tc::kBN;
    tc::gemm_tile(A, B, K, m0, n0, err, [&](int row, int col0, const float* v) {
        float4* dst = reinterpret_cast<float4*>(C + (size_t)row * N + col0);
#pragma unroll
        for (int i = 0; i < 4; ++i) dst[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    });
}

cudaError_t launch_gemm_bf16(int64_t M, int64_t N, int64_t K, const void* A, const void* B, float* C, int* err,
                             cudaStream_t st) {
    if (M <= 0 || N <= 0 || K <= 0) return cudaSuccess;
    if (M % tc::kBM || N % tc::kBN || K % tc::kBK) return cudaErrorInvalidValue;
    if (((uintptr_t)A | (uintptr_t)B | (uintptr_t)C) & 15u) return cudaErrorInvalidValue;
    if (M / tc::kBM > 65535 * 1024ll || N / tc::kBN > 65535) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSmemBytes);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)(M / tc::kBM), (unsigned)(N / tc::kBN));
    k_gemm_bf16<<<grid, tc::kThreads, tc::kSmemBytes, st>>>(reinterpret_cast<const __nv_bfloat16*>(A),
                                                             reinterpret_cast<const __nv_bfloat16*>(B), C, (int)N,
                                                             (int)K, err);
    return cudaGetLastError();
}

}  // namespace bqp
