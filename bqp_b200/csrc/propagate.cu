// sm_100a kernels of the batched propagator.
//
//   k_gravity   full-field gravity at Earth-fixed positions (force-eval API)
//   k_rhs       Encke force evaluation at given deviations (parity API)
//   k_propagate persistent one-trajectory-per-thread adaptive RK driver with
//               Encke rectification, fed by a device work queue
//
// The gravity coefficient table is staged once per CTA into shared memory
// (168 KB at degree 70) and read by warp-wide broadcasts.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.cuh"
#include "launch.h"
#include "traj.cuh"

namespace bqp {

// ----------------------------------------------------------------- kernels
template <int NT>
__global__ void __launch_bounds__(256, 1) k_gravity(GravTable T, int parts_max, int64_t n,
                                                    const double* __restrict__ pos, double* __restrict__ acc,
                                                    int32_t* __restrict__ status) {
    // rows are int-indexed inside a CTA: the launcher keeps each CTA's range
    // below 2^31 by running chunks
    const int64_t per_block = (n + gridDim.x - 1) / gridDim.x;
    const int64_t c0 = (int64_t)blockIdx.x * per_block;
    const int64_t c1 = c0 + per_block < n ? c0 + per_block : n;
    if (c0 >= c1) return;  // uniform across the CTA
    const double* p0 = pos + 3 * c0;
    double* a0 = acc + 3 * c0;
    int32_t* s0 = status ? status + c0 : nullptr;
    auto load = [&](int i, double& x, double& y, double& z) -> bool {
        const double ex = p0[3 * i], ey = p0[3 * i + 1], ez = p0[3 * i + 2];
        const double r2 = fma(ex, ex, fma(ey, ey, ez * ez));
        if (!(isfinite(r2) && r2 > 0.0)) {
            a0[3 * i] = a0[3 * i + 1] = a0[3 * i + 2] = NAN;
            if (s0) s0[i] = kGravityRadius;
            return false;
        }
        x = ex;
        y = ey;
        z = ez;
        return true;
    };
    auto store = [&](int i, const double* a, double x, double y, double z) {
        // add the C00 point mass back: the full field of the reference's
        // spherical_gravity_impl_frame_packed (gravity.rs:2638-2675)
        const double r2 = fma(x, x, fma(y, y, z * z));
        const double k = kMu / (r2 * sqrt(r2));
        a0[3 * i] = fma(-k, x, a[0]);
        a0[3 * i + 1] = fma(-k, y, a[1]);
        a0[3 * i + 2] = fma(-k, z, a[2]);
        if (s0) s0[i] = kOk;
    };
    auto lost = [&](int i) {
        a0[3 * i] = a0[3 * i + 1] = a0[3 * i + 2] = NAN;
        if (s0) s0[i] = kWatchdog;
    };
    gravity_cta<NT>(T, parts_max, (int)per_block, 0, (int)(c1 - c0), load, store, lost);
}

__global__ void k_rhs(const double* __restrict__ gtab, int ncells, int use_smem, ForceParams fp,
                      int64_t n, const double* __restrict__ equ, const double* __restrict__ seg_t0,
                      const double* __restrict__ jd0, const double* __restrict__ t,
                      const double* __restrict__ delta, const double* __restrict__ ballistic,
                      double am0, double cd0, double* __restrict__ out) {
    const double* tab = stage_table(gtab, ncells, use_smem != 0);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        Encke R;
        R.tab = tab;
        R.fp = &fp;
        R.base = baseline_new(equ + 6 * i);
        R.seg_t0 = seg_t0[i];
        R.jd0 = jd0[i];
        R.tai0 = 0.0;
        if (fp.frame.mode == 1 && !ft::tai_seconds_from_utc_jd(jd0[i], &R.tai0))
            R.tai0 = NAN;  // no segment: the evaluation returns NaN
        R.am = ballistic ? ballistic[2 * i] : am0;
        R.cd = ballistic ? ballistic[2 * i + 1] : cd0;
        R.side = -1;
        R.bad = 0;
        double d[6], o[6];
        for (int q = 0; q < 6; ++q) d[q] = delta[6 * i + q];
        R.eval(t[i], d, o);
        for (int q = 0; q < 6; ++q) out[6 * i + q] = o[q];
    }
}

// ------------------------------------------------- persistent work-queue kernel
// One trajectory per thread; a thread that finishes its trajectory pulls the
// next index from the device work queue (A.queue), so batches of uneven
// duration keep every lane busy.  Stage derivatives live in local memory.
template <int M>
__global__ void __launch_bounds__(256, 1) k_propagate(PropArgs A) {
    using T = Tab<M>;
    constexpr int S = T::S;
    const double* tab = stage_table(A.gtab, A.ncells, A.use_smem != 0);
    Encke R;
    R.tab = tab;
    R.fp = &A.force;
    R.side = -1;
    R.bad = 0;

    double k[S * 6];
    TrajState s;
    s.phase = kNeedTraj;
    s.s_idx = 0;
    int64_t traj = -1;
    const uint64_t t_launch = global_ns();
    bool timed_out = false;

    for (;;) {
        if (!timed_out && A.ctrl.max_kernel_ns > 0 && (int64_t)(global_ns() - t_launch) > A.ctrl.max_kernel_ns)
            timed_out = true;
        // ---- per-thread transitions (short, divergent)
        while (s.phase != kStepping) {
            if (s.phase == kNeedTraj || s.phase == kFinished) {
                const unsigned long long idx = atomicAdd(A.queue, 1ULL);
                if (idx >= (unsigned long long)A.n) {
                    s.phase = kDone;
                    break;
                }
                traj = (int64_t)idx;
                if (timed_out) {  // drain the queue: rows not started before the deadline
                    s.s_idx = 0;
                    s.steps = s.evals = 0;
                    traj_fail(A, s, traj, kWatchdog);
                    continue;
                }
                traj_begin(A, s, traj);
            }
            if (s.phase == kNeedSegment) seg_begin<M>(A, s, traj);
        }
        if (s.phase == kDone) break;

        const int32_t f0 = attempt_begin<M>(A, s, timed_out);
        if (f0 >= 0) {
            traj_fail(A, s, traj, f0);
            continue;
        }
        // ---- one step attempt (uniform across the warp)
        R.base = baseline_new(s.cur);
        R.seg_t0 = s.ct0;
        R.jd0 = s.jd0;
        R.tai0 = s.tai0;
        R.am = s.am;
        R.cd = s.cd;
        R.side = s.side;
        R.bad = 0;
        if (s.flags & kHaveK1) {
            for (int i = 0; i < 6; ++i) k[i] = s.k1c[i];
        } else {
            R.eval(s.t, s.y, k);
            ++s.evals;
        }
#pragma unroll 1
        for (int st = 1; st < S; ++st) {
            double yt[6];
            for (int i = 0; i < 6; ++i) yt[i] = s.y[i];
#pragma unroll 1
            for (int j = 0; j < st; ++j) {
                const double sc = s.hs * T::a(st, j);
                if (sc != 0.0)
                    for (int i = 0; i < 6; ++i) yt[i] = fma(k[j * 6 + i], sc, yt[i]);
            }
            R.eval(s.t + T::c(st) * s.hs, yt, k + st * 6);
            ++s.evals;
        }
        double ynext[6], err[6], err3[6];
        rk_combine<M>(s, [&](int st, int i) { return k[st * 6 + i]; }, ynext, err, err3);
        double en;
        int32_t code = -1;
        const int32_t d = attempt_decide<M>(A, s, k, ynext, err, err3, &en, &code);
        if (R.bad) {
            traj_fail(A, s, traj, R.bad == 3 ? kFrameTime : kGravityRadius);
            continue;
        }
        if (d == kFail) {
            traj_fail(A, s, traj, code);
            continue;
        }
        if (d == kAccept) {
            double dyn[6];
            const double* dy_next = nullptr;
            if (T::FSAL) {
                dy_next = k + (S - 1) * 6;
            } else if (s.flags & (kSegSampled | kEcl)) {
                R.eval(next_time(s), ynext, dyn);  // the reference's dense k1 (solver.rs:1672-1676)
                ++s.evals;
                dy_next = dyn;
            }
            attempt_accept<M>(A, s, traj, ynext, k, dy_next, en);
        }
    }
}

// --------------------------------------------------------------- launchers
static int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    }
    return n;
}

cudaError_t launch_gravity(const GravTable& T, int64_t n, const double* pos, double* acc, int32_t* status,
                           cudaStream_t st, int threads, int slots) {
    if (n <= 0) return cudaSuccess;
    const int nt = slots == 1 || slots == 2 ? slots : 4;
    auto ker = nt == 1 ? k_gravity<1> : (nt == 2 ? k_gravity<2> : k_gravity<4>);
    if (threads <= 0 || threads > 256) threads = 256;
    if (threads < 32) threads = 32;
    threads = threads / 32 * 32;
    int parts = kGravityPartsMax;
    size_t smem = gravity_smem_bytes(T, threads, nt, parts);
    if (smem > kSmemPerBlock) {
        parts = 1;
        smem = gravity_smem_bytes(T, threads, nt, parts);
    }
    cudaError_t e = cudaFuncSetAttribute(ker, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // one CTA per SM; each takes an equal share of the rows.  Chunks of at
    // most 2^30 rows keep a CTA's share int-indexed.
    const int64_t grid_cap = (int64_t)sm_count();
    const int64_t chunk = (int64_t)1 << 30;
    for (int64_t off = 0; off < n; off += chunk) {
        const int64_t m = n - off < chunk ? n - off : chunk;
        int64_t blocks = (m + 32 * nt - 1) / (32 * nt);
        if (blocks > grid_cap) blocks = grid_cap;
        ker<<<(unsigned)blocks, threads, smem, st>>>(T, parts, m, pos + 3 * off, acc + 3 * off,
                                                     status ? status + off : nullptr);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Space-weather drivers at n UTC Julian days, one per thread (the lookup the
// force kernels make at every evaluation): out[9 i] = F10 .. Y81c, dTc.
__global__ void k_jb_lookup(jb::DriverTable T, const double* __restrict__ jd, int64_t n, double* __restrict__ out,
                            int32_t* __restrict__ ok) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    jb::Drivers d;
    const bool found = jb::lookup_drivers(T, jd[i], &d);
    const double v[9] = {d.f10, d.f10b, d.s10, d.s10b, d.m10, d.m10b, d.y10, d.y10b, d.dtc};
    for (int k = 0; k < 9; ++k) out[9 * i + k] = found ? v[k] : NAN;
    ok[i] = found ? 1 : 0;
}

// Sun (body 0) / Moon (1) positions as the force kernels take them.
__global__ void k_body_positions(EphemTable E, int body, const double* __restrict__ jd, int64_t n,
                                 double* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (body == 0) sun_at(E, jd[i], out + 3 * i);
    else moon_at(E, jd[i], out + 3 * i);
}

cudaError_t launch_body_positions(const EphemTable& E, int body, const double* jd, int64_t n, double* out,
                                  cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int threads = 256;
    k_body_positions<<<(unsigned)((n + threads - 1) / threads), threads, 0, st>>>(E, body, jd, n, out);
    return cudaGetLastError();
}

cudaError_t launch_jb_lookup(const jb::DriverTable& T, const double* jd, int64_t n, double* out, int32_t* ok,
                             cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int threads = 256;
    k_jb_lookup<<<(unsigned)((n + threads - 1) / threads), threads, 0, st>>>(T, jd, n, out, ok);
    return cudaGetLastError();
}

cudaError_t launch_rhs(const double* gtab, int ncells, int use_smem, const ForceParams& fp, int64_t n,
                       const double* equ, const double* seg_t0, const double* jd0, const double* t,
                       const double* delta, const double* ballistic, double am0, double cd0,
                       double* out, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const size_t smem = use_smem ? (size_t)ncells * kCellDoubles * sizeof(double) : 0;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_rhs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int threads = 256;
    int64_t blocks = (n + threads - 1) / threads;
    const int64_t cap = (int64_t)sm_count();
    if (blocks > cap) blocks = cap;
    k_rhs<<<(unsigned)blocks, threads, smem, st>>>(gtab, ncells, use_smem, fp, n, equ, seg_t0, jd0, t, delta,
                                                   ballistic, am0, cd0, out);
    return cudaGetLastError();
}

template <int M>
static cudaError_t launch_prop_m(const PropArgs& A, int threads, int blocks, cudaStream_t st) {
    const size_t smem = A.use_smem ? (size_t)A.ncells * kCellDoubles * sizeof(double) : 0;
    cudaError_t e = cudaFuncSetAttribute(k_propagate<M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(smem > 0 ? smem : 0));
    if (e != cudaSuccess) return e;
    k_propagate<M><<<blocks, threads, smem, st>>>(A);
    return cudaGetLastError();
}

cudaError_t launch_propagate(const PropArgs& A, int method, int threads, int blocks, cudaStream_t st) {
    if (A.n <= 0) return cudaSuccess;
    if (threads <= 0) threads = 256;
    if (threads > 256) threads = 256;
    if (blocks <= 0) {
        const int64_t want = (A.n + threads - 1) / threads;
        blocks = (int)(want < sm_count() ? want : sm_count());
        if (blocks < 1) blocks = 1;
    }
    switch (method) {
        case kDopri5: return launch_prop_m<kDopri5>(A, threads, blocks, st);
        case kDop853: return launch_prop_m<kDop853>(A, threads, blocks, st);
        case kDopri5Compat: return launch_prop_m<kDopri5Compat>(A, threads, blocks, st);
        case kVern7: return launch_prop_m<kVern7>(A, threads, blocks, st);
        case kVern9: return launch_prop_m<kVern9>(A, threads, blocks, st);
        default: return cudaErrorInvalidValue;
    }
}

int device_sm_count() { return sm_count(); }

}  // namespace bqp
