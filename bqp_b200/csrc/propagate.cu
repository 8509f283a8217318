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

#define BQP_TAB_CONST static __constant__ const
#include "kernels.cuh"
#include "launch.h"
#include "rk_tableaus.h"

namespace bqp {

// ------------------------------------------------------------ table staging
// Copy the field table into dynamic shared memory with 16-byte vector loads.
__device__ __forceinline__ const double* stage_table(const double* __restrict__ g, int ncells,
                                                     bool to_smem) {
    extern __shared__ __align__(16) double smem_tab[];
    if (!to_smem) return g;
    const int nvec = ncells * (kCellDoubles / 2);
    const double2* src = reinterpret_cast<const double2*>(g);
    double2* dst = reinterpret_cast<double2*>(smem_tab);
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) dst[i] = __ldg(src + i);
    __syncthreads();
    return smem_tab;
}

// ----------------------------------------------------------------- kernels
__global__ void k_gravity(const double* __restrict__ gtab, int order, int ncells, int use_smem,
                          int64_t n, const double* __restrict__ pos, double* __restrict__ acc,
                          int32_t* __restrict__ status) {
    const double* tab = stage_table(gtab, ncells, use_smem != 0);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
        const double r2 = fma(x, x, fma(y, y, z * z));
        double a[3];
        if (!(isfinite(r2) && r2 > 0.0)) {
            a[0] = a[1] = a[2] = NAN;
            if (status) status[i] = kGravityRadius;
        } else {
            gravity_field(tab, order, x, y, z, a);
            // add the C00 point mass back: the full field of the reference's
            // spherical_gravity_impl_frame_packed (gravity.rs:2638-2675)
            const double k = kMu / (r2 * sqrt(r2));
            a[0] = fma(-k, x, a[0]);
            a[1] = fma(-k, y, a[1]);
            a[2] = fma(-k, z, a[2]);
            if (status) status[i] = kOk;
        }
        acc[3 * i] = a[0];
        acc[3 * i + 1] = a[1];
        acc[3 * i + 2] = a[2];
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

// ------------------------------------------------------------- RK tableaus
template <int M>
struct Tab;
template <>
struct Tab<kDopri5> {
    static constexpr int S = 7, ORDER_ERR = 4, FSAL = 1, HAS_E3 = 0;
    __device__ static double a(int i, int j) { return bqp_dopri5_a[i * S + j]; }
    __device__ static double b(int i) { return bqp_dopri5_b[i]; }
    __device__ static double c(int i) { return bqp_dopri5_c[i]; }
    __device__ static double e(int i) { return bqp_dopri5_e[i]; }
    __device__ static double e3(int) { return 0.0; }
};
template <>
struct Tab<kDopri5Compat> : Tab<kDopri5> {};
template <>
struct Tab<kDop853> {
    static constexpr int S = 12, ORDER_ERR = 5, FSAL = 0, HAS_E3 = 1;
    __device__ static double a(int i, int j) { return bqp_dop853_a[i * S + j]; }
    __device__ static double b(int i) { return bqp_dop853_b[i]; }
    __device__ static double c(int i) { return bqp_dop853_c[i]; }
    __device__ static double e(int i) { return bqp_dop853_e[i]; }
    __device__ static double e3(int i) { return bqp_dop853_e3[i]; }
};

// ---------------------------------------------------------- the RK driver
// Output modes of k_propagate.
enum OutMode : int32_t { kOutFinalEci = 0, kOutSampledEci = 1, kOutSampledDelta = 2 };

enum Phase : int32_t { kNeedTraj = 0, kNeedSegment = 1, kStepping = 2, kDone = 3 };

__device__ __forceinline__ bool finite6(const double* v) {
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 6; ++i) ok = ok && isfinite(v[i]);
    return ok;
}

__device__ __forceinline__ double clampd(double x, double lo, double hi) {
    return fmin(fmax(x, lo), hi);
}

// Sampled output writer: deviation at sample time ts on the current segment
// baseline -> deviation against the original baseline (integrator.rs:1163-1177)
// or the ECI state (lib.rs:316-322).
__device__ __forceinline__ void write_sample(const PropArgs& A, int64_t traj, int s_idx,
                                             const double* dseg, double ts, const Baseline& seg,
                                             double seg_t0, const Baseline& orig, double orig_t0,
                                             bool had) {
    double* o = A.out + ((size_t)traj * A.n_t + s_idx) * 6;
    double bo[6];
    baseline_state(orig, ts - orig_t0, bo);
    double dorig[6];
    if (had) {
        double bs[6];
        baseline_state(seg, ts - seg_t0, bs);
        for (int i = 0; i < 6; ++i) dorig[i] = (dseg[i] + bs[i]) - bo[i];
    } else {
        for (int i = 0; i < 6; ++i) dorig[i] = dseg[i];
    }
    if (A.out_mode == kOutSampledDelta) {
        for (int i = 0; i < 6; ++i) o[i] = dorig[i];
    } else {
        for (int i = 0; i < 6; ++i) o[i] = bo[i] + dorig[i];
    }
}

template <int M>
__global__ void __launch_bounds__(256, 1) k_propagate(PropArgs A) {
    using T = Tab<M>;
    constexpr int S = T::S;
    const double* tab = stage_table(A.gtab, A.ncells, A.use_smem != 0);
    const bool sampled = A.out_mode != kOutFinalEci;
    const double order = (double)T::ORDER_ERR + 1.0;
    const double inv_order = 1.0 / order;
    const CtrlParams& C = A.ctrl;

    Encke R;
    R.tab = tab;
    R.fp = &A.force;
    R.bad = 0;

    double k[S * 6];  // stage derivatives (local memory)
    double y[6], k1c[6];
    double equ0[6], cur[6];
    Baseline orig;
    int64_t traj = -1;
    int32_t phase = kNeedTraj;
    double t0 = A.t0, tf = 0.0, ct0 = 0.0, seg_tf = 0.0, t = 0.0, h = 0.0;
    double err_prev = 0.0, t_comp = 0.0;
    bool have_prev = false, just_rej = false, have_k1 = false, had = false;
    int64_t seg_steps = 0, steps = 0, evals = 0, attempts = 0, restarts = 0, max_restarts = 0;
    int32_t rejects = 0;
    int s_idx = 0;
    const uint64_t t_launch = global_ns();
    bool timed_out = false;

    for (;;) {
        if (!timed_out && C.max_kernel_ns > 0 && (int64_t)(global_ns() - t_launch) > C.max_kernel_ns)
            timed_out = true;
        // ---- per-thread transitions (short, divergent)
        while (phase != kStepping) {
            if (phase == kNeedTraj) {
                const unsigned long long idx = atomicAdd(A.queue, 1ULL);
                if (idx >= (unsigned long long)A.n) {
                    phase = kDone;
                    break;
                }
                traj = (int64_t)idx;
                if (timed_out) {
                    // drain the queue: rows not started before the deadline
                    A.status[traj] = kWatchdog;
                    if (A.steps) A.steps[traj] = 0;
                    if (A.evals) A.evals[traj] = 0;
                    const int nout = sampled ? A.n_t : 1;
                    for (int q = 0; q < 6 * nout; ++q) A.out[(size_t)traj * 6 * nout + q] = NAN;
                    continue;
                }
                tf = A.tf[traj];
                R.jd0 = A.epoch[traj];
                R.am = A.ballistic ? A.ballistic[2 * traj] : A.am0;
                R.cd = A.ballistic ? A.ballistic[2 * traj + 1] : A.cd0;
                bool ok;
                if (A.input_equinoctial) {
                    for (int i = 0; i < 6; ++i) equ0[i] = A.in[6 * traj + i];
                    ok = baseline_new(equ0).ok != 0 && finite6(equ0);
                } else {
                    double e[6];
                    for (int i = 0; i < 6; ++i) e[i] = A.in[6 * traj + i];
                    ok = finite6(e) && eci_to_equinoctial(e, equ0);
                }
                ok = ok && isfinite(tf) && isfinite(R.jd0) && tf >= t0;
                steps = evals = attempts = restarts = 0;
                had = false;
                s_idx = 0;
                if (!ok) {
                    A.status[traj] = kInvalidInput;
                    if (A.steps) A.steps[traj] = 0;
                    if (A.evals) A.evals[traj] = 0;
                    const int nout = sampled ? A.n_t : 1;
                    for (int q = 0; q < 6 * nout; ++q) A.out[(size_t)traj * 6 * nout + q] = NAN;
                    continue;  // next trajectory
                }
                orig = baseline_new(equ0);
                for (int i = 0; i < 6; ++i) cur[i] = equ0[i];
                ct0 = t0;
                const double span = fabs(tf - t0);
                int64_t mr = (int64_t)ceil(span / (C.h_max > 0.0 ? C.h_max : 1.0)) + 128;
                max_restarts = mr < 100 ? 100 : (mr > 500000 ? 500000 : mr);
                // the sampled path stops after 100 segments (integrator.rs:2366, 2408-2414)
                if (sampled) max_restarts = 100;
                if (sampled) {
                    // samples at the arc start carry a zero deviation
                    const double zero[6] = {0, 0, 0, 0, 0, 0};
                    while (s_idx < A.n_t && A.t_eval[s_idx] <= t0) {
                        write_sample(A, traj, s_idx, zero, A.t_eval[s_idx], orig, t0, orig, t0, false);
                        ++s_idx;
                    }
                }
                phase = kNeedSegment;
            }
            if (phase == kNeedSegment) {
                int32_t fin = -1;
                if (had && fabs(tf - ct0) < 1e-12) fin = kOk;  // integrator.rs:3440-3452
                else if (restarts >= max_restarts) fin = sampled ? kMaxSteps : kRestartBudget;
                if (fin >= 0) {
                    if (!sampled) {
                        double* o = A.out + 6 * traj;
                        if (fin == kOk) {
                            double ce[6], ob[6];
                            equinoctial_to_eci(cur, 0.0, ce);
                            baseline_state(orig, tf - t0, ob);
                            for (int i = 0; i < 6; ++i) o[i] = ob[i] + (ce[i] - ob[i]);
                        } else {
                            for (int i = 0; i < 6; ++i) o[i] = NAN;
                        }
                    } else if (fin != kOk) {
                        for (int q = s_idx; q < A.n_t; ++q)
                            for (int i = 0; i < 6; ++i) A.out[((size_t)traj * A.n_t + q) * 6 + i] = NAN;
                    }
                    A.status[traj] = fin;
                    if (A.steps) A.steps[traj] = steps;
                    if (A.evals) A.evals[traj] = evals;
                    phase = kNeedTraj;
                    continue;
                }
                ++restarts;
                const double rem = tf - ct0;
                seg_tf = fabs(rem) > kMaxSegmentS ? ct0 + kMaxSegmentS : tf;
                R.base = baseline_new(cur);
                R.seg_t0 = ct0;
                R.bad = 0;
                t = ct0;
                for (int i = 0; i < 6; ++i) y[i] = 0.0;
                const double span = fabs(seg_tf - ct0);
                double hmax = fabs(C.h_max);
                if (!isfinite(hmax) || hmax <= 0.0) hmax = span;
                if (M == kDopri5Compat) {
                    h = clampd(fabs((seg_tf - ct0) / 100.0), 1e-3, fmax(fmax(hmax, 1e-10), 1e-3));
                } else {
                    h = clampd(span <= 60.0 ? span / 2.0 : span / 100.0, C.h_min, hmax);
                }
                err_prev = 0.0;
                t_comp = 0.0;
                have_prev = just_rej = false;
                have_k1 = false;
                rejects = 0;
                seg_steps = 0;
                if (M == kDopri5Compat) {
                    R.eval(t, y, k1c);
                    ++evals;
                    have_k1 = true;
                }
                phase = kStepping;
                if (!(span > 0.0)) {
                    // zero-length segment: the deviation stays zero
                    phase = kNeedSegment;
                    had = true;
                    ct0 = seg_tf;
                }
            }
        }
        if (phase == kDone) break;

        // ---- one step attempt (uniform across the warp)
        const double hmax = fabs(C.h_max) > 0.0 && isfinite(C.h_max) ? fabs(C.h_max) : fabs(seg_tf - ct0);
        const double hmin = M == kDopri5Compat ? 1e-10 : C.h_min;
        const double rem = seg_tf - t;
        double hs = fabs(h) < fabs(rem) ? h : rem;
        const bool lands = hs == rem;
        int32_t fail = -1;
        if (seg_steps >= C.max_steps) fail = kMaxSteps;
        else if (M != kDopri5Compat && fabs(hs) < hmin && !lands) fail = kStepUnderflow;
        else if (++attempts > C.max_attempts || timed_out) fail = kWatchdog;
        double ynext[6], err[6], err3[6];
        if (fail < 0) {
            if (have_k1) {
                for (int i = 0; i < 6; ++i) k[i] = k1c[i];
            } else {
                R.eval(t, y, k);
                ++evals;
            }
#pragma unroll 1
            for (int st = 1; st < S; ++st) {
                double yt[6];
#pragma unroll
                for (int i = 0; i < 6; ++i) yt[i] = y[i];
#pragma unroll 1
                for (int j = 0; j < st; ++j) {
                    const double sc = hs * T::a(st, j);
                    if (sc != 0.0) {
#pragma unroll
                        for (int i = 0; i < 6; ++i) yt[i] = fma(k[j * 6 + i], sc, yt[i]);
                    }
                }
                R.eval(t + T::c(st) * hs, yt, k + st * 6);
                ++evals;
            }
            double comp[6], comp3[6];
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                ynext[i] = y[i];
                err[i] = 0.0;
                err3[i] = 0.0;
                comp[i] = 0.0;
                comp3[i] = 0.0;
            }
#pragma unroll 1
            for (int st = 0; st < S; ++st) {
                const double hb = hs * T::b(st), he = hs * T::e(st), he3 = hs * T::e3(st);
                if (hb != 0.0) {
#pragma unroll
                    for (int i = 0; i < 6; ++i) ynext[i] = fma(k[st * 6 + i], hb, ynext[i]);
                }
                if (he != 0.0) {
#pragma unroll
                    for (int i = 0; i < 6; ++i) {  // Kahan-compensated (solver.rs:2120-2150)
                        const double yk = he * k[st * 6 + i] - comp[i];
                        const double acc = err[i] + yk;
                        comp[i] = (acc - err[i]) - yk;
                        err[i] = acc;
                    }
                }
                if (T::HAS_E3 && he3 != 0.0) {
#pragma unroll
                    for (int i = 0; i < 6; ++i) {
                        const double yk = he3 * k[st * 6 + i] - comp3[i];
                        const double acc = err3[i] + yk;
                        comp3[i] = (acc - err3[i]) - yk;
                        err3[i] = acc;
                    }
                }
            }
            if (M == kDopri5Compat) {
                ++seg_steps;  // the compat loop counts attempts (lightyear_compat.rs)
                ++steps;
            }
        }

        // ---- step control (short, divergent)
        bool seg_done = false;
        if (fail < 0) {
            const double dir_h = fabs(hs);
            double en = NAN, thr = 1.0;
            bool finite_step = finite6(ynext) && finite6(err);
            if (finite_step) {
                if (M == kDopri5Compat || !C.scaled) {
                    double m5 = 0.0, m3 = 0.0;
                    for (int i = 0; i < 6; ++i) {
                        m5 = fmax(m5, fabs(err[i]));
                        m3 = fmax(m3, fabs(err3[i]));
                    }
                    const bool use_e3 = T::HAS_E3 && M != kDopri5Compat && C.eps >= 1e-6;
                    en = use_e3 ? sqrt(fma(m5, m5, 0.01 * m3 * m3)) : m5;
                    thr = C.eps;
                } else {
                    double s5 = 0.0, s3 = 0.0;
                    for (int i = 0; i < 6; ++i) {
                        const double sc = C.atol + C.rtol * fmax(fabs(y[i]), fabs(ynext[i]));
                        const double dn = sc > 0.0 ? sc : C.atol;
                        const double e5 = err[i] / dn, e3 = err3[i] / dn;
                        s5 = fma(e5, e5, s5);
                        s3 = fma(e3, e3, s3);
                    }
                    const double r5 = sqrt(s5 / 6.0);
                    if (T::HAS_E3) {
                        const double r3 = sqrt(s3 / 6.0);
                        en = sqrt(fma(r5, r5, 0.01 * r3 * r3));
                    } else {
                        en = r5;
                    }
                    thr = 1.0;
                }
            }
            if (!finite_step || !isfinite(en)) {
                ++rejects;
                have_k1 = M == kDopri5Compat ? have_k1 : false;
                if (rejects > C.max_rejects) fail = kNonFinite;
                h = clampd(dir_h * 0.1, hmin, M == kDopri5Compat ? fmax(hmax, 1e-10) : hmax);
            } else if (en <= thr || dir_h <= hmin) {
                double tn;
                if (lands) {
                    tn = seg_tf;
                } else {
                    const double ky = hs - t_comp;
                    const double nx = t + ky;
                    t_comp = (nx - t) - ky;
                    tn = nx;
                }
                if (!isfinite(tn)) {
                    fail = kNonFinite;
                } else {
                    if (M != kDopri5Compat) {
                        ++seg_steps;
                        ++steps;
                    }
                    rejects = 0;
                    double dy_prev[6], dy_next[6];
                    for (int i = 0; i < 6; ++i) dy_prev[i] = k[i];
                    if (T::FSAL) {
                        for (int i = 0; i < 6; ++i) k1c[i] = k[(S - 1) * 6 + i];
                        have_k1 = true;
                    } else if (sampled) {
                        R.eval(tn, ynext, k1c);
                        ++evals;
                        have_k1 = true;
                    } else {
                        have_k1 = false;
                    }
                    for (int i = 0; i < 6; ++i) dy_next[i] = k1c[i];
                    if (sampled) {
                        while (s_idx < A.n_t) {
                            const double ts = A.t_eval[s_idx];
                            if (ts - tn > 0.0) break;
                            double ds[6];
                            if (ts == tn) {
                                for (int i = 0; i < 6; ++i) ds[i] = ynext[i];
                            } else {
                                const double hd = tn - t;
                                const double tau = clampd((ts - t) / hd, 0.0, 1.0);
                                const double t2 = tau * tau, t3 = t2 * tau;
                                const double h00 = 2.0 * t3 - 3.0 * t2 + 1.0, h10 = t3 - 2.0 * t2 + tau;
                                const double h01 = -2.0 * t3 + 3.0 * t2, h11 = t3 - t2;
                                for (int i = 0; i < 6; ++i)
                                    ds[i] = h00 * y[i] + h10 * hd * dy_prev[i] + h01 * ynext[i] +
                                            h11 * hd * dy_next[i];
                            }
                            write_sample(A, traj, s_idx, ds, ts, R.base, ct0, orig, t0, had);
                            ++s_idx;
                        }
                    }
                    t = tn;
                    for (int i = 0; i < 6; ++i) y[i] = ynext[i];
                    // PI controller, accept branch (solver.rs:445-506; compat: lightyear_compat.rs)
                    const double eff = en > 0.0 ? en : thr * 0.1;
                    double factor;
                    if (M == kDopri5Compat) {
                        factor = (have_prev && err_prev > 0.0)
                                     ? 0.9 * pow(C.eps / eff, 0.7 / 5.0) * pow(err_prev / C.eps, 0.4 / 5.0)
                                     : 0.9 * pow(C.eps / eff, 0.2);
                        const double mg = just_rej ? 2.0 : 5.0;
                        h = clampd(dir_h * clampd(factor, 0.2, mg), 1e-10, fmax(hmax, 1e-10));
                    } else {
                        if (!C.scaled) {
                            factor = (have_prev && err_prev > 0.0)
                                         ? 0.9 * pow(C.eps / eff, 0.7 / order) * pow(err_prev / C.eps, 0.4 / order)
                                         : 0.9 * pow(C.eps / eff, inv_order);
                        } else {
                            factor = (have_prev && err_prev > 0.0)
                                         ? 0.9 * pow(1.0 / eff, 0.7 / order) * pow(err_prev, 0.4 / order)
                                         : 0.9 * pow(eff, -inv_order);
                        }
                        const double mgb = fmin(1.0 + 4.0 * (5.0 / order), 5.0);
                        const double mg = just_rej ? fmin(mgb, 2.0) : mgb;
                        h = clampd(dir_h * clampd(factor, 0.2, mg), hmin, hmax);
                    }
                    err_prev = en;
                    have_prev = true;
                    just_rej = false;
                    if (A.force.ground_check) {
                        double bs[6];
                        baseline_state(R.base, t - ct0, bs);
                        const double alt = geodetic_altitude_km(bs[0] + y[0], bs[1] + y[1], bs[2] + y[2],
                                                                A.force.earth_radius);
                        if (!(alt >= kGroundAltitudeKm)) fail = kGround;
                    }
                    if (fail < 0 && t == seg_tf) seg_done = true;
                }
            } else {
                ++rejects;
                if (M != kDopri5Compat) have_k1 = false;
                if (rejects > C.max_rejects) {
                    fail = kMaxRejects;
                } else if (M == kDopri5Compat) {
                    const double factor = 0.9 * pow(C.eps / en, 0.2);
                    h = clampd(dir_h * clampd(factor, 0.1, 0.5), 1e-10, fmax(hmax, 1e-10));
                    err_prev = en;
                    have_prev = true;
                    just_rej = true;
                } else {
                    const double factor = !C.scaled ? 0.9 * pow(C.eps / en, inv_order) : 0.9 * pow(en, -inv_order);
                    h = clampd(dir_h * clampd(factor, 0.1, 0.5), hmin, hmax);
                    just_rej = true;
                }
            }
        }
        if (fail < 0 && R.bad) fail = kGravityRadius;
        if (fail < 0 && seg_done) {
            // rectification (integrator.rs:941-979)
            const double dsq = fma(y[0], y[0], fma(y[1], y[1], y[2] * y[2]));
            if (dsq > kRebaseKm * kRebaseKm || seg_tf != tf) {
                double bs[6], e[6], ne[6];
                baseline_state(R.base, seg_tf - ct0, bs);
                for (int i = 0; i < 6; ++i) e[i] = bs[i] + y[i];
                if (!eci_to_equinoctial(e, ne)) {
                    fail = kRebaseFailed;
                } else {
                    for (int i = 0; i < 6; ++i) cur[i] = ne[i];
                    ct0 = seg_tf;
                    had = true;
                    phase = kNeedSegment;
                }
            } else {
                // arc complete on this segment
                if (!sampled) {
                    double* o = A.out + 6 * traj;
                    double ob[6];
                    baseline_state(orig, tf - t0, ob);
                    if (had) {
                        double bs[6];
                        baseline_state(R.base, tf - ct0, bs);
                        for (int i = 0; i < 6; ++i) o[i] = ob[i] + ((y[i] + bs[i]) - ob[i]);
                    } else {
                        for (int i = 0; i < 6; ++i) o[i] = ob[i] + y[i];
                    }
                }
                A.status[traj] = kOk;
                if (A.steps) A.steps[traj] = steps;
                if (A.evals) A.evals[traj] = evals;
                phase = kNeedTraj;
            }
        }
        if (fail >= 0) {
            if (!sampled) {
                for (int i = 0; i < 6; ++i) A.out[6 * traj + i] = NAN;
            } else {
                for (int q = s_idx; q < A.n_t; ++q)
                    for (int i = 0; i < 6; ++i) A.out[((size_t)traj * A.n_t + q) * 6 + i] = NAN;
            }
            A.status[traj] = fail;
            if (A.steps) A.steps[traj] = steps;
            if (A.evals) A.evals[traj] = evals;
            phase = kNeedTraj;
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
                           const double* pos, double* acc, int32_t* status, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const size_t smem = use_smem ? (size_t)ncells * kCellDoubles * sizeof(double) : 0;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k_gravity, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int threads = 256;
    int64_t blocks = (n + threads - 1) / threads;
    const int64_t cap = (int64_t)sm_count() * 2;
    if (blocks > cap) blocks = cap;
    k_gravity<<<(unsigned)blocks, threads, smem, st>>>(gtab, order, ncells, use_smem, n, pos, acc, status);
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
