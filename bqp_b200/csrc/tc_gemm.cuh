// BF16 tensor-core GEMM on the 5th-generation tensor cores (tcgen05):
//
//     C[M x N] (FP32) = A[M x K] (BF16, row-major) * B[N x K]^T (BF16, row-major)
//
// One CTA of 128 threads computes a 128 x 256 tile of C; its FP32 accumulator
// lives in tensor memory (256 columns of the SM's 512).  K is staged 64 at a
// time into shared memory, double-buffered, in the canonical K-major layout
// without swizzle: 8-row x 16-byte core matrices, core matrices of one
// 8-row group consecutive along K.  One elected thread issues the four
// K = 16 MMAs of a stage and commits them to the stage's mbarrier; the
// threads refill a buffer only after its MMAs have completed.  The epilogue
// reads the accumulator back with tcgen05.ld (warp w owns TMEM lanes
// 32w..32w+31, i.e. rows 32w..32w+31 of the tile).
//
// Requirements (checked by the launcher): M % 128 == 0, N % 256 == 0,
// K % 64 == 0, 16-byte aligned rows.  Every wait is bounded (1 s of
// %globaltimer); a CTA that times out records it in *err, still releases its
// tensor memory and returns.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"

namespace bqp {
namespace tc {

constexpr int kBM = 128, kBN = 256, kBK = 64;
constexpr int kThreads = 128;
constexpr int kTmemCols = 256;
constexpr uint64_t kWaitNs = 1000000000ull;

// bytes of one stage: A 128 x 64 and B 256 x 64 BF16
constexpr int kStageA = kBM * kBK * 2, kStageB = kBN * kBK * 2;
constexpr int kSmemBytes = 2 * (kStageA + kStageB) + 64;

// element (r, k) of a rows x 64 K-major tile, in BF16 elements
__device__ __forceinline__ int tile_index(int r, int k) {
    return ((r >> 3) * (kBK / 8) + (k >> 3)) * 64 + (r & 7) * 8 + (k & 7);
}

// shared-memory matrix descriptor (sm100: version 1, no swizzle)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= 1ull << 46;  // descriptor version for sm100
    return d;         // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// instruction descriptor of kind::f16: FP32 accumulate, BF16 A and B, both
// K-major, M = 128, N = kBN
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kBN >> 3) << 17) |
                            ((uint32_t)(kBM >> 4) << 24);

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    const uint64_t t0 = global_ns();
    for (uint32_t it = 0;; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 255u) == 255u && global_ns() - t0 > kWaitNs) return false;
    }
}

// Stage k-chunk kc of A (rows m0..m0+127) and B (rows n0..n0+255) into the
// tile buffers: 16-byte global loads, 16-byte shared stores.
__device__ __forceinline__ void load_stage(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B,
                                           int K, int m0, int n0, int kc, __nv_bfloat16* sa, __nv_bfloat16* sb) {
    // a 16-byte vector = 8 consecutive k of one row = one core-matrix row
    for (int v = threadIdx.x; v < kBM * (kBK / 8); v += kThreads) {
        const int r = v / (kBK / 8), k8 = (v % (kBK / 8)) * 8;
        const uint4 x = *reinterpret_cast<const uint4*>(A + (size_t)(m0 + r) * K + kc + k8);
        *reinterpret_cast<uint4*>(sa + tile_index(r, k8)) = x;
    }
    for (int v = threadIdx.x; v < kBN * (kBK / 8); v += kThreads) {
        const int r = v / (kBK / 8), k8 = (v % (kBK / 8)) * 8;
        const uint4 x = *reinterpret_cast<const uint4*>(B + (size_t)(n0 + r) * K + kc + k8);
        *reinterpret_cast<uint4*>(sb + tile_index(r, k8)) = x;
    }
}

// The tile loop.  epi(row, col0, v[16]) receives 16 consecutive FP32 results
// of one row (col0 = first column of C).
template <class Epilogue>
__device__ __forceinline__ void gemm_tile(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B,
                                          int K, int m0, int n0, int* err, Epilogue epi) {
    extern __shared__ __align__(128) unsigned char tc_smem[];
    __nv_bfloat16* sa[2] = {reinterpret_cast<__nv_bfloat16*>(tc_smem),
                            reinterpret_cast<__nv_bfloat16*>(tc_smem + kStageA + kStageB)};
    __nv_bfloat16* sb[2] = {reinterpret_cast<__nv_bfloat16*>(tc_smem + kStageA),
                            reinterpret_cast<__nv_bfloat16*>(tc_smem + 2 * kStageA + kStageB)};
    uint64_t* bars = reinterpret_cast<uint64_t*>(tc_smem + 2 * (kStageA + kStageB));  // 2 mbarriers
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
    const uint32_t bar_a[2] = {(uint32_t)__cvta_generic_to_shared(&bars[0]),
                               (uint32_t)__cvta_generic_to_shared(&bars[1])};
    const int warp = threadIdx.x >> 5;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(tmem_slot)),
                     "r"((uint32_t)kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a[0]) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a[1]) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    const int nk = K / kBK;
    uint32_t phase[2] = {0, 0};
    bool pending[2] = {false, false};  // a commit on this buffer's barrier not yet seen complete
    bool ok = true;
    for (int s = 0; s < nk && ok; ++s) {
        const int buf = s & 1;
        if (s >= 2) {  // the MMAs that read this buffer two stages ago
            // one verdict for the CTA, so every thread takes the same path
            ok = __syncthreads_and(mbar_wait(bar_a[buf], phase[buf]));
            if (!ok) break;
            phase[buf] ^= 1u;
            pending[buf] = false;
        }
        load_stage(A, B, K, m0, n0, s * kBK, sa[buf], sb[buf]);
        // make the generic-proxy stores visible to the tensor cores
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = (uint32_t)__cvta_generic_to_shared(sa[buf]);
            const uint32_t b0 = (uint32_t)__cvta_generic_to_shared(sb[buf]);
#pragma unroll
            for (int kk = 0; kk < kBK; kk += 16) {
                // two 8-wide K chunks per MMA: LBO = next chunk (128 B),
                // SBO = next 8-row group (kBK / 8 core matrices of 128 B)
                const uint64_t da = smem_desc(a0 + (kk / 8) * 128, 128, (kBK / 8) * 128);
                const uint64_t db = smem_desc(b0 + (kk / 8) * 128, 128, (kBK / 8) * 128);
                const uint32_t acc = (s > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(kIdesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             bar_a[buf])
                         : "memory");
        }
        pending[buf] = true;
    }
    // drain: the last one or two commits
    if (ok) {
        for (int s = (nk >= 2 ? nk - 2 : 0); s < nk && ok; ++s) {
            const int buf = s & 1;
            ok = __syncthreads_and(mbar_wait(bar_a[buf], phase[buf]));
            if (!ok) break;
            phase[buf] ^= 1u;
            pending[buf] = false;
        }
    }
    if (!ok) {
        if (threadIdx.x == 0) {
            atomicExch(err, 1);
            // keep shared and tensor memory until the MMAs issued on them
            // have completed, each for at most the same bound
            for (int b = 0; b < 2; ++b)
                if (pending[b]) mbar_wait(bar_a[b], phase[b]);
        }
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int row = warp * 32 + (threadIdx.x & 31);
        const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < kBN; c0 += 16) {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
                "%13, %14, %15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(lane_addr + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            float v[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
            epi(m0 + row, n0 + c0, v);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTmemCols)
                     : "memory");
}

}  // namespace tc
}  // namespace bqp
