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
__global__ void k_gravity(const double* __restrict__ gtab, int order, int ncells, int use_smem, int64_t n,
                          const double* __restrict__ pos, double* __restrict__ acc, int32_t* __restrict__ status) {
    const int64_t per_block = (n + gridDim.x - 1) / gridDim.x;
    const int64_t b0 = (int64_t)blockIdx.x * per_block;
    const int64_t b1 = b0 + per_block < n ? b0 + per_block : n;
    if (b0 >= b1) return;  // uniform across the CTA
    const double* tab = stage_table(gtab, ncells, use_smem != 0);
    for (int64_t base = b0; base < b1; base += (int64_t)blockDim.x * NT) {
        double px[NT], py[NT], pz[NT], a[NT][3];
        int64_t idx[NT];
        bool on[NT];
#pragma unroll
        for (int q = 0; q < NT; ++q) {
            idx[q] = base + (int64_t)q * blockDim.x + threadIdx.x;
            on[q] = idx[q] < b1;
            px[q] = 7000.0;
            py[q] = 0.0;
            pz[q] = 0.0;
            if (on[q]) {
                const int64_t i = idx[q];
                const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
                const double r2 = fma(x, x, fma(y, y, z * z));
                if (!(isfinite(r2) && r2 > 0.0)) {
                    acc[3 * i] = acc[3 * i + 1] = acc[3 * i + 2] = NAN;
                    if (status) status[i] = kGravityRadius;
                    on[q] = false;
                } else {
                    px[q] = x;
                    py[q] = y;
                    pz[q] = z;
                }
            }
        }
        gravity_field_multi<NT>(tab, order, px, py, pz, a);
#pragma unroll
        for (int q = 0; q < NT; ++q) {
            if (!on[q]) continue;
            const int64_t i = idx[q];
            // add the C00 point mass back: the full field of the reference's
            // spherical_gravity_impl_frame_packed (gravity.rs:2638-2675)
            const double r2 = fma(px[q], px[q], fma(py[q], py[q], pz[q] * pz[q]));
            const double k = kMu / (r2 * sqrt(r2));
            acc[3 * i] = fma(-k, px[q], a[q][0]);
            acc[3 * i + 1] = fma(-k, py[q], a[q][1]);
            acc[3 * i + 2] = fma(-k, pz[q], a[q][2]);
            if (status) status[i] = kOk;
        }
    }
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
        R.am = ballistic ? ballistic[2 * i] : am0;
        R.cd = ballistic ? ballistic[2 * i + 1] : cd0;
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
        R.am = s.am;
        R.cd = s.cd;
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
            traj_fail(A, s, traj, kGravityRadius);
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
            } else if (s.flags & kSegSampled) {
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

cudaError_t launch_gravity(const double* gtab, int order, int ncells, int use_smem, int64_t n,
                           const double* pos, double* acc, int32_t* status, cudaStream_t st, int threads,
                           int slots) {
    if (n <= 0) return cudaSuccess;
    const size_t smem = use_smem ? (size_t)ncells * kCellDoubles * sizeof(double) : 0;
    const int nt = slots == 1 || slots == 4 ? slots : 2;
    auto ker = nt == 1 ? k_gravity<1> : (nt == 4 ? k_gravity<4> : k_gravity<2>);
    cudaError_t e = cudaFuncSetAttribute(ker, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (threads <= 0) threads = 256;
    int64_t blocks = (n + (int64_t)threads * nt - 1) / ((int64_t)threads * nt);
    const int64_t cap = (int64_t)sm_count() * (use_smem ? 1 : 4);
    if (blocks > cap) blocks = cap;
    ker<<<(unsigned)blocks, threads, smem, st>>>(gtab, order, ncells, use_smem, n, pos, acc, status);
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
        default: return cudaErrorInvalidValue;
    }
}

int device_sm_count() { return sm_count(); }

}  // namespace bqp
