// Both forms of the eclipse crossing scan on given Hermite paths: the
// per-thread walk (persistent engine) and the warp-cooperative walk
// (stage-synchronous engine).  bqp_ecl_scan_check runs them for its tests.
#include <cuda_runtime.h>

#include "eclipse.cuh"
#include "launch.h"

namespace bqp {

namespace {

// path row: p0[3], v0[3], p1[3], v1[3], t0, t1, from, jd0; result row:
// status, found, old side, new side (as doubles), t_old, t_new, bound
__device__ void load_path(const double* r, EclPath* H, double* from, double* jd0) {
    for (int i = 0; i < 3; ++i) {
        H->p0[i] = r[i];
        H->v0[i] = r[3 + i];
        H->p1[i] = r[6 + i];
        H->v1[i] = r[9 + i];
    }
    H->t0 = r[12];
    H->t1 = r[13];
    *from = r[14];
    *jd0 = r[15];
}

__device__ void store_result(double* o, int32_t e, bool found, const EclBracket& br) {
    o[0] = e;
    o[1] = found ? 1.0 : 0.0;
    o[2] = found ? br.old_side : 0.0;
    o[3] = found ? br.new_side : 0.0;
    o[4] = found ? br.t_old : 0.0;
    o[5] = found ? br.t_new : 0.0;
    o[6] = found ? br.bound : 0.0;
}

__global__ void k_scan_serial(ForceParams fp, int64_t n, const double* __restrict__ paths, double* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    EclPath H;
    double from, jd0;
    load_path(paths + 16 * i, &H, &from, &jd0);
    const EclGeo G{&fp, jd0};
    bool found = false;
    EclBracket br{};
    const int32_t e = ecl_first_crossing(G, H, from, H.t1, &found, &br);
    store_result(out + 7 * i, e, found, br);
}

__global__ void __launch_bounds__(256) k_scan_warp(ForceParams fp, int64_t n, const double* __restrict__ paths,
                                                   double* __restrict__ out) {
    __shared__ EclWarpStore ws[8];
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= n) return;  // uniform across the warp
    EclPath H;
    double from, jd0;
    load_path(paths + 16 * i, &H, &from, &jd0);
    const EclGeo G{&fp, jd0};
    bool found = false;
    EclBracket br{};
    const int32_t e = ecl_first_crossing_warp(G, H, from, H.t1, ws[threadIdx.x >> 5], &found, &br);
    if ((threadIdx.x & 31) == 0) store_result(out + 7 * i, e, found, br);
}

}  // namespace

cudaError_t launch_ecl_scan(const ForceParams& fp, int64_t n, const double* paths, double* out, int warp,
                            cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (warp) {
        const int64_t blocks = (n * 32 + 255) / 256;
        k_scan_warp<<<(unsigned)blocks, 256, 0, st>>>(fp, n, paths, out);
    } else {
        k_scan_serial<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(fp, n, paths, out);
    }
    return cudaGetLastError();
}

}  // namespace bqp
