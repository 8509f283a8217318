// One CTA's share of a gravity batch, used by the gravity-only kernel and by
// the stage-synchronous engine's gravity stage.
//
// The table (8 doubles per cell) sits in shared memory; each cell read puts
// 64 bytes into every lane's registers, so a thread carries NT rows to share
// those reads.  A batch of a few hundred rows per SM then needs only a few
// warps, too few to hide latency on their own, so the CTA is cut into
// `parts` groups of `tpart` threads: every group evaluates all rows of a
// pass over its own run of columns (cut to about equal cell counts), and the
// groups' partial sums are added in shared memory in a fixed order.
#pragma once
#include "gravity.cuh"
#include "kernels.cuh"

namespace bqp {

// opt-in shared memory per CTA, less room for the static mbarrier
constexpr size_t kSmemPerBlock = 227 * 1024 - 64;
constexpr uint64_t kStageWaitNs = 1000000000ull;   // 1 s bound on the table copy
constexpr uint64_t kStageDrainNs = 2000000000ull;  // after a timeout: 2 s more for the copy to land

// Sticky flag of this translation unit's gravity kernels: set when a CTA's
// table copy did not land within kStageWaitNs.  Every later CTA (of this and
// later launches) then stages nothing and reports its rows lost, so no CTA
// starts on an SM where an earlier CTA's copy may still be writing shared
// memory.  It stays set until the process exits: a bulk copy that takes
// seconds means the device is not in a state to trust.
static __device__ unsigned int g_stage_fault = 0u;

// Copy `bytes` (a multiple of 16; both addresses 16-byte aligned) from global
// to shared memory with the bulk-copy engine, completion signalled on an
// mbarrier.  Thread 0 issues the copy; every thread waits for at most
// kStageWaitNs; all get false if any thread saw the copy unfinished then.
// On that failure the CTA sets g_stage_fault and thread 0 keeps the CTA
// resident for up to kStageDrainNs more, until the copy has landed, so the
// CTA does not exit with its copy in flight unless the copy never completes.
__device__ __forceinline__ bool bulk_stage(void* smem_dst, const void* gsrc, uint32_t bytes) {
    __shared__ __align__(8) uint64_t bar;
    const uint32_t bar_a = (uint32_t)__cvta_generic_to_shared(&bar);
    const uint32_t dst_a = (uint32_t)__cvta_generic_to_shared(smem_dst);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // one read of the sticky flag decides for the whole CTA
    const bool faulted =
        __syncthreads_or(threadIdx.x == 0 && *static_cast<volatile unsigned int*>(&g_stage_fault) != 0u);
    if (faulted) return false;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a), "r"(bytes) : "memory");
        constexpr uint32_t kChunk = 32768;
        for (uint32_t off = 0; off < bytes; off += kChunk) {
            const uint32_t n = bytes - off < kChunk ? bytes - off : kChunk;
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    dst_a + off),
                "l"(static_cast<const char*>(gsrc) + off), "r"(n), "r"(bar_a)
                : "memory");
        }
    }
    uint32_t done = 0;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 0;; ++it) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\tselp.u32 %0, 1, 0, "
            "p;\n\t}"
            : "=r"(done)
            : "r"(bar_a)
            : "memory");
        if (done) break;
        if ((it & 255u) == 255u && global_ns() - t0 > kStageWaitNs) break;
    }
    // one verdict for the whole CTA (a thread may give up just before the
    // copy lands while another sees it land)
    if (!__syncthreads_or(done == 0)) return true;
    if (threadIdx.x == 0) {
        atomicExch(&g_stage_fault, 1u);
        const uint64_t t1 = global_ns();
        for (uint32_t it = 0;; ++it) {
            uint32_t landed;
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\tselp.u32 %0, 1, "
                "0, p;\n\t}"
                : "=r"(landed)
                : "r"(bar_a)
                : "memory");
            if (landed) break;
            if ((it & 255u) == 255u && global_ns() - t1 > kStageDrainNs) break;
        }
    }
    __syncthreads();
    return false;
}
constexpr int kGravityPartsMax = 4;

struct GravLayout {
    int tpart;  // threads per group (a multiple of 32, at most the CTA)
    int parts;  // groups
};

BQP_HD GravLayout gravity_layout(int rows, int nt, int block, int parts_max) {
    const int need = (rows + nt - 1) / nt;
    int tpart = (need + 31) / 32 * 32;
    if (tpart > block) tpart = block;
    if (tpart < 32) tpart = 32;
    int parts = block / tpart;
    if (parts > parts_max) parts = parts_max;
    if (parts < 1) parts = 1;
    return {tpart, parts};
}

// The field table as the gravity kernels see it.  Plain form: `tab` holds
// the FP64 cells of every column.  Split form (ls > 0): `tab` holds the FP64
// cells of rows <= ls followed by the FP32 cells of the rest
// (gravity_columns_split).
struct GravTable {
    const double* tab;
    int order;
    int ls;          // 0: plain FP64; else the last FP64 row
    uint32_t bytes;  // size of tab
    int in_smem;     // 1: staged into shared memory per CTA
};

inline uint32_t gravity_table_bytes(int order, int ls) {
    if (ls <= 0) return (uint32_t)gravity_cells(order) * kCellDoubles * sizeof(double);
    return (uint32_t)(split_lo_cells(ls) * kCellDoubles * sizeof(double) +
                      split_hi_cells(order, ls) * kCellDoubles * sizeof(float));
}

// Dynamic shared memory of a CTA of `block` threads: the table (if staged)
// plus the partial-sum area of groups 1..parts-1.
inline size_t gravity_smem_bytes(const GravTable& T, int block, int nt, int parts_max) {
    const size_t tab = T.in_smem ? T.bytes : 0;
    const size_t red = parts_max > 1 ? (size_t)(block - 32) * nt * 3 * sizeof(double) : 0;
    return tab + red;
}

// Rows [b0, b1) of this CTA; the layout (and so the order in which a row's
// column sums are added) follows layout_rows, the same for every CTA of a
// launch, so a row's result does not depend on which CTA it lands in.
// load(i, x, y, z) fetches row i's Earth-fixed
// position and returns false for a row to leave out (it records that row's
// outcome itself; every group calls it, so it must be idempotent).
// store(i, a, x, y, z) receives the field of row i (group 0 only).
// lost(i) records that row i got no field because the table copy did not
// complete in time.
template <int NT, class Load, class Store, class Lost>
__device__ __forceinline__ void gravity_cta(const GravTable& T, int parts_max, int layout_rows, int b0, int b1,
                                            Load load, Store store, Lost lost) {
    extern __shared__ __align__(16) double smem_dyn[];
    const GravLayout L = gravity_layout(layout_rows, NT, blockDim.x, parts_max);
    if (T.in_smem && !bulk_stage(smem_dyn, T.tab, T.bytes)) {
        for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) lost(i);
        return;  // the verdict is the same in every thread
    }
    const int order = T.order;
    const double* __restrict__ gtab = T.tab;
    double* red = smem_dyn + (T.in_smem ? T.bytes / sizeof(double) : 0);
    const int part = threadIdx.x / L.tpart;
    const int tid = threadIdx.x - part * L.tpart;
    const bool member = part < L.parts;
    const int j0 = gravity_part_column(order, part, L.parts);
    const int j1 = gravity_part_column(order, part + 1, L.parts);
    const int per_pass = L.tpart * NT;
    for (int base = b0; base < b1; base += per_pass) {
        double px[NT], py[NT], pz[NT], a[NT][3];
        bool on[NT];
#pragma unroll
        for (int q = 0; q < NT; ++q) {
            const int i = base + q * L.tpart + tid;
            px[q] = 7000.0;  // a valid dummy position for idle lanes
            py[q] = 0.0;
            pz[q] = 0.0;
            on[q] = member && i < b1 && load(i, px[q], py[q], pz[q]);
        }
        if (member) {
            if (T.ls > 0) {
                const size_t lo_doubles = (size_t)split_lo_cells(T.ls) * kCellDoubles;
                if (T.in_smem)
                    gravity_columns_split<NT>(smem_dyn, reinterpret_cast<const float*>(smem_dyn + lo_doubles),
                                              order, T.ls, j0, j1, px, py, pz, a);
                else
                    gravity_columns_split<NT>(gtab, reinterpret_cast<const float*>(gtab + lo_doubles), order,
                                              T.ls, j0, j1, px, py, pz, a);
            } else {
                if (T.in_smem)
                    gravity_columns<NT>(smem_dyn, order, j0, j1, px, py, pz, a);
                else
                    gravity_columns<NT>(gtab, order, j0, j1, px, py, pz, a);
            }
        }
        if (L.parts > 1) {
            if (member && part > 0) {
#pragma unroll
                for (int q = 0; q < NT; ++q)
                    for (int c = 0; c < 3; ++c)
                        red[((size_t)(part - 1) * per_pass + q * L.tpart + tid) * 3 + c] = a[q][c];
            }
            __syncthreads();
            if (part == 0) {
                for (int g = 1; g < L.parts; ++g) {
#pragma unroll
                    for (int q = 0; q < NT; ++q)
                        for (int c = 0; c < 3; ++c)
                            a[q][c] += red[((size_t)(g - 1) * per_pass + q * L.tpart + tid) * 3 + c];
                }
            }
            __syncthreads();  // the area is reused by the next pass
        }
        if (part == 0) {
#pragma unroll
            for (int q = 0; q < NT; ++q)
                if (on[q]) store(base + q * L.tpart + tid, a[q], px[q], py[q], pz[q]);
        }
    }
}

}  // namespace bqp
