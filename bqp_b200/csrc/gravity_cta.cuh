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

namespace bqp {

constexpr size_t kSmemPerBlock = 227 * 1024;  // opt-in dynamic shared memory per CTA
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

// Dynamic shared memory of a CTA of `block` threads: the table (if staged)
// plus the partial-sum area of groups 1..parts-1.
inline size_t gravity_smem_bytes(int ncells, bool table_in_smem, int block, int nt, int parts_max) {
    const size_t tab = table_in_smem ? (size_t)ncells * kCellDoubles * sizeof(double) : 0;
    const size_t red = parts_max > 1 ? (size_t)(block - 32) * nt * 3 * sizeof(double) : 0;
    return tab + red;
}

// Rows [b0, b1) of this CTA.  load(i, x, y, z) fetches row i's Earth-fixed
// position and returns false for a row to leave out (it records that row's
// outcome itself; every group calls it, so it must be idempotent).
// store(i, a, x, y, z) receives the field of row i (group 0 only).
template <int NT, class Load, class Store>
__device__ __forceinline__ void gravity_cta(const double* __restrict__ gtab, int order, int ncells, bool table_in_smem,
                                            int parts_max, int b0, int b1, Load load, Store store) {
    extern __shared__ __align__(16) double smem_dyn[];
    const GravLayout L = gravity_layout(b1 - b0, NT, blockDim.x, parts_max);
    if (table_in_smem) {
        const int nvec = ncells * (kCellDoubles / 2);
        const double2* src = reinterpret_cast<const double2*>(gtab);
        double2* dst = reinterpret_cast<double2*>(smem_dyn);
        for (int i = threadIdx.x; i < nvec; i += blockDim.x) dst[i] = __ldg(src + i);
    }
    double* red = smem_dyn + (table_in_smem ? (size_t)ncells * kCellDoubles : 0);
    __syncthreads();
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
            if (table_in_smem)
                gravity_columns<NT>(smem_dyn, order, j0, j1, px, py, pz, a);
            else
                gravity_columns<NT>(gtab, order, j0, j1, px, py, pz, a);
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
