// Per-trajectory controller shared by both propagation engines: the
// persistent work-queue kernel (k_propagate) and the stage-synchronous
// pipeline (pipeline.cu).  It carries the reference's solver semantics once:
//
//   explicit RK step bookkeeping, Kahan-compensated error sums and time
//   (odesolve/solver.rs:1965-2173, 1551-1572), max-norm / WRMS error with the
//   DOP853 3rd-order blend (1431-1520), the PI controller (445-531), the
//   DOPRI5 compatibility loop's own controller (lightyear_compat.rs), Encke
//   segments of at most 5400 s with a rebase when |dr| > 10 km or the segment
//   is not the last (integrator.rs:941-979, 3418-3560), the restart budget
//   ceil(span/dt_max)+128 clamped to [100, 500000] (3912-3917), the sampled
//   path's 100-segment cap (2366, 2408-2414) and its Hermite samples
//   (solver.rs:1746-1800).
#pragma once
#include <cstdint>

#include "eclipse.cuh"
#include "kernels.cuh"
#include "launch.h"

#ifndef BQP_TAB_CONST
#define BQP_TAB_CONST static __constant__ const
#endif
#include "rk_tableaus.h"

namespace bqp {

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

template <>
struct Tab<kVern7> {
    static constexpr int S = 10, ORDER_ERR = 6, FSAL = 0, HAS_E3 = 0;
    __device__ static double a(int i, int j) { return bqp_vern7_a[i * S + j]; }
    __device__ static double b(int i) { return bqp_vern7_b[i]; }
    __device__ static double c(int i) { return bqp_vern7_c[i]; }
    __device__ static double e(int i) { return bqp_vern7_e[i]; }
    __device__ static double e3(int) { return 0.0; }
};

template <>
struct Tab<kVern9> {
    static constexpr int S = 16, ORDER_ERR = 8, FSAL = 0, HAS_E3 = 0;
    __device__ static double a(int i, int j) { return bqp_vern9_a[i * S + j]; }
    __device__ static double b(int i) { return bqp_vern9_b[i]; }
    __device__ static double c(int i) { return bqp_vern9_c[i]; }
    __device__ static double e(int i) { return bqp_vern9_e[i]; }
    __device__ static double e3(int) { return 0.0; }
};

enum OutMode : int32_t { kOutFinalEci = 0, kOutSampledEci = 1, kOutSampledDelta = 2 };
enum Phase : int32_t { kNeedTraj = 0, kNeedSegment = 1, kStepping = 2, kDone = 3, kFinished = 4 };
// kEcl: the row runs through the binary-eclipse coordinator (SRP on).
enum Flag : int32_t { kHavePrev = 1, kJustRej = 2, kHaveK1 = 4, kHad = 8, kLands = 16, kSegSampled = 32, kEcl = 64 };

struct TrajState {
    double tf, ct0, seg_tf, t, h, err_prev, t_comp, hs, hcarry;
    double jd0, am, cd;
    double tai0;   // continuous TAI seconds of t = 0 (IAU frame), 0 otherwise
    double lhmax;  // the eclipse leg's maximum step
    double cur[6], equ0[6], y[6], k1c[6];
    int32_t flags, rejects, s_idx, phase, status;
    int32_t side;  // the eclipse leg's fixed side (1 shadow, 0 lit), -1 without SRP
    int64_t seg_steps, steps, evals, attempts, restarts, max_restarts;
};

__device__ __forceinline__ bool finite6(const double* v) {
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 6; ++i) ok = ok && isfinite(v[i]);
    return ok;
}

__device__ __forceinline__ double clampd(double x, double lo, double hi) { return fmin(fmax(x, lo), hi); }

__device__ __forceinline__ bool sampled_mode(const PropArgs& A) { return A.out_mode != kOutFinalEci; }

// ---------------------------------------------------------------- outputs
// Deviation at sample time ts on the segment baseline -> deviation against
// the original baseline (integrator.rs:1163-1177) or ECI (lib.rs:316-322).
static __device__ __noinline__ void write_sample(const PropArgs& A, const TrajState& s, int64_t traj,
                                          const double* dseg, double ts) {
    double* o = A.out + ((size_t)traj * A.n_t + s.s_idx) * 6;
    const Baseline orig = baseline_new(s.equ0);
    double bo[6];
    baseline_state(orig, ts - A.t0, bo);
    double dorig[6];
    if (s.flags & kHad) {
        double bs[6];
        baseline_state(baseline_new(s.cur), ts - s.ct0, bs);
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

__device__ __forceinline__ void write_counters(const PropArgs& A, int64_t traj, const TrajState& s) {
    A.status[traj] = s.status;
    if (A.steps) A.steps[traj] = s.steps;
    if (A.evals) A.evals[traj] = s.evals;
}

// Fail a trajectory: NaN-fill what is not yet written (batch.rs:297).
static __device__ __noinline__ void traj_fail(const PropArgs& A, TrajState& s, int64_t traj, int32_t code) {
    if (!sampled_mode(A)) {
        for (int i = 0; i < 6; ++i) A.out[6 * traj + i] = NAN;
    } else {
        for (int q = s.s_idx; q < A.n_t; ++q)
            for (int i = 0; i < 6; ++i) A.out[((size_t)traj * A.n_t + q) * 6 + i] = NAN;
    }
    s.status = code;
    s.phase = kFinished;
    write_counters(A, traj, s);
}

// Successful end of the arc with the last segment's deviation d at tf.
static __device__ __noinline__ void traj_finish_with(const PropArgs& A, TrajState& s, int64_t traj, const double* d) {
    if (!sampled_mode(A)) {
        double* o = A.out + 6 * traj;
        double ob[6];
        baseline_state(baseline_new(s.equ0), s.tf - A.t0, ob);
        if (s.flags & kHad) {
            double bs[6];
            baseline_state(baseline_new(s.cur), s.tf - s.ct0, bs);
            for (int i = 0; i < 6; ++i) o[i] = ob[i] + ((d[i] + bs[i]) - ob[i]);
        } else {
            for (int i = 0; i < 6; ++i) o[i] = ob[i] + d[i];
        }
    }
    s.status = kOk;
    s.phase = kFinished;
    write_counters(A, traj, s);
}

// ------------------------------------------------------------ transitions
// Load trajectory `traj` from the inputs.  Leaves phase kNeedSegment, or
// kFinished with an invalid-input status.
static __device__ __noinline__ void traj_begin(const PropArgs& A, TrajState& s, int64_t traj) {
    s.tf = A.tf[traj];
    s.jd0 = A.epoch[traj];
    s.am = A.ballistic ? A.ballistic[2 * traj] : A.am0;
    s.cd = A.ballistic ? A.ballistic[2 * traj + 1] : A.cd0;
    s.steps = s.evals = s.attempts = s.restarts = 0;
    s.seg_steps = 0;
    s.flags = 0;
    s.hcarry = 0.0;
    s.rejects = 0;
    s.s_idx = 0;
    s.status = kOk;
    bool ok;
    if (A.input_equinoctial) {
        for (int i = 0; i < 6; ++i) s.equ0[i] = A.in[6 * traj + i];
        ok = finite6(s.equ0) && baseline_new(s.equ0).ok != 0;
    } else {
        double e[6];
        for (int i = 0; i < 6; ++i) e[i] = A.in[6 * traj + i];
        ok = finite6(e) && eci_to_equinoctial(e, s.equ0);
    }
    ok = ok && isfinite(s.tf) && isfinite(s.jd0) && s.tf >= A.t0;
    if (!ok) {
        traj_fail(A, s, traj, kInvalidInput);
        return;
    }
    // the IAU frame's time origin (rhs.rs:2754): a UTC epoch before the
    // integer-leap era has none, and the first Earth-fixed evaluation fails
    s.tai0 = 0.0;
    if (A.force.frame.mode == 1 && (A.force.gravity_on || A.force.drag) &&
        !ft::tai_seconds_from_utc_jd(s.jd0, &s.tai0)) {
        traj_fail(A, s, traj, kFrameTime);
        return;
    }
    for (int i = 0; i < 6; ++i) s.cur[i] = s.equ0[i];
    s.ct0 = A.t0;
    s.side = -1;
    s.lhmax = 0.0;
    if (A.force.srp && A.force.cr > 0.0 && A.force.p_sun > 0.0 && s.am > 0.0) {
        // SRP in effect (rhs.rs:31-36): the eclipse coordinator, whose
        // samples are always carried to the original baseline
        EclState& E = A.ecl[traj];
        E = EclState{};
        s.flags |= kEcl | kHad;
        if (s.tf != A.t0) {
            const Baseline b0 = baseline_new(s.cur);
            const double zero[6] = {0, 0, 0, 0, 0, 0};
            if (!ecl_envelope(b0, s.ct0, zero, s.ct0)) {
                traj_fail(A, s, traj, kEclEnvelope);
                return;
            }
            const EclGeo G{&A.force, s.jd0};
            int side;
            double margin;
            if (int32_t e = ecl_side_at(G, b0, s.ct0, zero, s.ct0, &side, &margin)) {
                traj_fail(A, s, traj, e);
                return;
            }
            s.side = side;
        }
    }
    const double span = fabs(s.tf - A.t0);
    const int64_t mr = (int64_t)ceil(span / (A.ctrl.h_max > 0.0 ? A.ctrl.h_max : 1.0)) + 128;
    s.max_restarts = mr < 100 ? 100 : (mr > 500000 ? 500000 : mr);
    if (sampled_mode(A)) {
        s.max_restarts = 100;
        const double zero[6] = {0, 0, 0, 0, 0, 0};
        while (s.s_idx < A.n_t && A.t_eval[s.s_idx] <= A.t0) {
            write_sample(A, s, traj, zero, A.t_eval[s.s_idx]);
            ++s.s_idx;
        }
    }
    s.phase = kNeedSegment;
}

// Start the next Encke segment, or end the arc.  Leaves kStepping or
// kFinished.
template <int M>
__device__ void ecl_seg_begin(const PropArgs& A, TrajState& s, int64_t traj);

template <int M>
__device__ __noinline__ void seg_begin(const PropArgs& A, TrajState& s, int64_t traj) {
    if (s.flags & kEcl) {
        ecl_seg_begin<M>(A, s, traj);
        return;
    }
    for (int guard = 0; guard < 2 && s.phase == kNeedSegment; ++guard) {
        if ((s.flags & kHad) && fabs(s.tf - s.ct0) < 1e-12) {  // integrator.rs:3440-3452
            const double zero[6] = {0, 0, 0, 0, 0, 0};
            traj_finish_with(A, s, traj, zero);
            return;
        }
        if (s.restarts >= s.max_restarts) {
            traj_fail(A, s, traj, sampled_mode(A) ? kMaxSteps : kRestartBudget);
            return;
        }
        ++s.restarts;
        const double rem = s.tf - s.ct0;
        s.seg_tf = fabs(rem) > kMaxSegmentS ? s.ct0 + kMaxSegmentS : s.tf;
        const double span = fabs(s.seg_tf - s.ct0);
        if (!(span > 0.0)) {
            s.flags |= kHad;
            s.ct0 = s.seg_tf;
            continue;
        }
        s.t = s.ct0;
        for (int i = 0; i < 6; ++i) s.y[i] = 0.0;
        double hmax = fabs(A.ctrl.h_max);
        if (!isfinite(hmax) || hmax <= 0.0) hmax = span;
        // A segment holding samples runs the reference's sampled solver
        // (integrate_segment_with_method: dense first-stage reuse, and the
        // previous sampled segment's final step as h0 when dt_max > 60 s,
        // integrator.rs:187-216); one without samples runs the final-state
        // solver (integrate_final_no_events_with_rhs, h0 = None).
        const bool seg_sampled = sampled_mode(A) && s.s_idx < A.n_t && A.t_eval[s.s_idx] <= s.seg_tf + 1e-9;
        if (M == kDopri5Compat)
            s.h = clampd(fabs((s.seg_tf - s.ct0) / 100.0), 1e-3, fmax(fmax(hmax, 1e-10), 1e-3));
        else if (seg_sampled && s.hcarry > 0.0 && A.ctrl.h_max > 60.0)
            s.h = clampd(s.hcarry, A.ctrl.h_min, hmax);
        else
            s.h = clampd(span <= 60.0 ? span / 2.0 : span / 100.0, A.ctrl.h_min, hmax);
        s.err_prev = 0.0;
        s.t_comp = 0.0;
        s.flags &= kHad;  // clear controller memory and the reusable first stage
        if (seg_sampled) s.flags |= kSegSampled;
        s.rejects = 0;
        s.seg_steps = 0;
        s.phase = kStepping;
    }
}

// The end time of the current attempt, as attempt_accept computes it
// (Kahan-compensated unless the step lands on the segment end).
__device__ __forceinline__ double next_time(const TrajState& s) {
    if (s.flags & kLands) return s.seg_tf;
    return s.t + (s.hs - s.t_comp);
}

__device__ __forceinline__ double seg_hmax(const PropArgs& A, const TrajState& s) {
    if (s.flags & kEcl) return s.lhmax;
    const double hm = fabs(A.ctrl.h_max);
    return (hm > 0.0 && isfinite(hm)) ? hm : fabs(s.seg_tf - s.ct0);
}

// Size the next attempt (hs, lands) or fail it.  Returns -1 or a status.
template <int M>
__device__ __forceinline__ int32_t attempt_begin(const PropArgs& A, TrajState& s, bool timed_out) {
    const double hmin = M == kDopri5Compat ? 1e-10 : A.ctrl.h_min;
    const double rem = s.seg_tf - s.t;
    s.hs = fabs(s.h) < fabs(rem) ? s.h : rem;
    if (s.hs == rem) s.flags |= kLands;
    else s.flags &= ~kLands;
    if (s.seg_steps >= A.ctrl.max_steps) return kMaxSteps;
    if (M != kDopri5Compat && fabs(s.hs) < hmin && !(s.flags & kLands)) return kStepUnderflow;
    if (++s.attempts > A.ctrl.max_attempts || timed_out) return kWatchdog;
    if (M == kDopri5Compat) {  // the compat loop counts attempts (lightyear_compat.rs)
        ++s.seg_steps;
        ++s.steps;
    }
    return -1;
}

// ynext and the Kahan-compensated error estimates from the stage
// derivatives K(st, i) (solver.rs:2098-2172).
template <int M, typename KAt>
__device__ __forceinline__ void rk_combine(const TrajState& s, KAt K, double* ynext, double* err, double* err3) {
    using T = Tab<M>;
    double comp[6], comp3[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        ynext[i] = s.y[i];
        err[i] = err3[i] = comp[i] = comp3[i] = 0.0;
    }
#pragma unroll 1
    for (int st = 0; st < T::S; ++st) {
        const double hb = s.hs * T::b(st), he = s.hs * T::e(st), he3 = s.hs * T::e3(st);
        if (hb == 0.0 && he == 0.0 && he3 == 0.0) continue;
        double kv[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) kv[i] = K(st, i);
        if (hb != 0.0) {
#pragma unroll
            for (int i = 0; i < 6; ++i) ynext[i] = fma(kv[i], hb, ynext[i]);
        }
        if (he != 0.0) {
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                const double yk = he * kv[i] - comp[i];
                const double acc = err[i] + yk;
                comp[i] = (acc - err[i]) - yk;
                err[i] = acc;
            }
        }
        if (T::HAS_E3 && he3 != 0.0) {
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                const double yk = he3 * kv[i] - comp3[i];
                const double acc = err3[i] + yk;
                comp3[i] = (acc - err3[i]) - yk;
                err3[i] = acc;
            }
        }
    }
}

enum Decision : int32_t { kReject = 0, kAccept = 1, kFail = 2 };

// Error norm and accept / reject (solver.rs:1413-1540 and the reject branch
// 1880-1905; the compat loop's own branches).  On reject it updates h and
// returns kReject; on failure it returns kFail with *code set.
template <int M>
__device__ __forceinline__ int32_t attempt_decide(const PropArgs& A, TrajState& s, const double* y0_k,
                                                  const double* ynext, const double* err, const double* err3,
                                                  double* en_out, int32_t* code) {
    using T = Tab<M>;
    const CtrlParams& C = A.ctrl;
    const double order = (double)T::ORDER_ERR + 1.0;
    const double inv_order = 1.0 / order;
    const double hmin = M == kDopri5Compat ? 1e-10 : C.h_min;
    const double hmax = seg_hmax(A, s);
    const double hmax_c = M == kDopri5Compat ? fmax(hmax, 1e-10) : hmax;
    const double ah = fabs(s.hs);
    double en = NAN, thr = 1.0;
    const bool finite_step = finite6(ynext) && finite6(err);
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
                const double sc = C.atol + C.rtol * fmax(fabs(s.y[i]), fabs(ynext[i]));
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
        }
    }
    *en_out = en;
    if (!finite_step || !isfinite(en)) {
        ++s.rejects;
        if (M == kDopri5Compat) {
            for (int i = 0; i < 6; ++i) s.k1c[i] = y0_k[i];
            s.flags |= kHaveK1;
        } else {
            s.flags &= ~kHaveK1;
        }
        if (s.rejects > C.max_rejects) {
            *code = kNonFinite;
            return kFail;
        }
        s.h = clampd(ah * 0.1, hmin, hmax_c);
        return kReject;
    }
    if (en <= thr || ah <= hmin) return kAccept;
    ++s.rejects;
    if (M == kDopri5Compat) {
        for (int i = 0; i < 6; ++i) s.k1c[i] = y0_k[i];
        s.flags |= kHaveK1;
    } else {
        s.flags &= ~kHaveK1;
    }
    if (s.rejects > C.max_rejects) {
        *code = kMaxRejects;
        return kFail;
    }
    if (M == kDopri5Compat) {
        const double factor = 0.9 * pow(C.eps / en, 0.2);
        s.h = clampd(ah * clampd(factor, 0.1, 0.5), 1e-10, hmax_c);
        s.err_prev = en;
        s.flags |= kHavePrev | kJustRej;
    } else {
        const double factor = !C.scaled ? 0.9 * pow(C.eps / en, inv_order) : 0.9 * pow(en, -inv_order);
        s.h = clampd(ah * clampd(factor, 0.1, 0.5), hmin, hmax);
        s.flags |= kJustRej;
    }
    return kReject;
}

// Samples inside the accepted step [s.t, tn]: the step's cubic Hermite
// interpolant (solver.rs:1746-1800), the end state itself at tn.
static __device__ __noinline__ void emit_samples(const PropArgs& A, TrajState& s, int64_t traj, double tn,
                                                 const double* ynext, const double* dy_prev, const double* dy_next) {
    while (s.s_idx < A.n_t) {
        const double ts = A.t_eval[s.s_idx];
        if (ts - tn > 0.0) break;
        double ds[6];
        if (ts == tn) {
            for (int i = 0; i < 6; ++i) ds[i] = ynext[i];
        } else {
            const double hd = tn - s.t;
            const double tau = clampd((ts - s.t) / hd, 0.0, 1.0);
            const double t2 = tau * tau, t3 = t2 * tau;
            const double h00 = 2.0 * t3 - 3.0 * t2 + 1.0, h10 = t3 - 2.0 * t2 + tau;
            const double h01 = -2.0 * t3 + 3.0 * t2, h11 = t3 - t2;
            for (int i = 0; i < 6; ++i)
                ds[i] = h00 * s.y[i] + h10 * hd * dy_prev[i] + h01 * ynext[i] + h11 * hd * dy_next[i];
        }
        write_sample(A, s, traj, ds, ts);
        ++s.s_idx;
    }
}

template <int M>
__device__ __noinline__ void ecl_accept(const PropArgs& A, TrajState& s, int64_t traj, const double* ynext,
                           const double* dy_prev, const double* dy_next, double en);

// Accepted step: time update, samples, PI controller, ground check and the
// segment end.  dy_prev = derivative at the step start, dy_next = at its end
// (FSAL last stage or the dense stage; may be null in final-state mode).
template <int M>
__device__ __noinline__ void attempt_accept(const PropArgs& A, TrajState& s, int64_t traj, const double* ynext,
                                            const double* dy_prev, const double* dy_next, double en) {
    using T = Tab<M>;
    if (M != kDopri5Compat && (s.flags & kEcl)) {
        ecl_accept<M>(A, s, traj, ynext, dy_prev, dy_next, en);
        return;
    }
    const CtrlParams& C = A.ctrl;
    const double order = (double)T::ORDER_ERR + 1.0;
    const double inv_order = 1.0 / order;
    const double hmin = M == kDopri5Compat ? 1e-10 : C.h_min;
    const double hmax = seg_hmax(A, s);
    const double ah = fabs(s.hs);
    double tn;
    if (s.flags & kLands) {
        tn = s.seg_tf;
    } else {
        const double ky = s.hs - s.t_comp;
        const double nx = s.t + ky;
        s.t_comp = (nx - s.t) - ky;
        tn = nx;
    }
    if (!isfinite(tn)) {
        traj_fail(A, s, traj, kNonFinite);
        return;
    }
    if (M != kDopri5Compat) {
        ++s.seg_steps;
        ++s.steps;
    }
    s.rejects = 0;
    if (sampled_mode(A)) emit_samples(A, s, traj, tn, ynext, dy_prev, dy_next);
    if (T::FSAL || (s.flags & kSegSampled)) {
        for (int i = 0; i < 6; ++i) s.k1c[i] = dy_next[i];
        s.flags |= kHaveK1;
    } else {
        s.flags &= ~kHaveK1;
    }
    s.t = tn;
    for (int i = 0; i < 6; ++i) s.y[i] = ynext[i];
    const double thr = (M == kDopri5Compat || !C.scaled) ? C.eps : 1.0;
    const double eff = en > 0.0 ? en : thr * 0.1;
    const bool have_prev = (s.flags & kHavePrev) && s.err_prev > 0.0;
    const bool just_rej = s.flags & kJustRej;
    double factor;
    if (M == kDopri5Compat) {
        factor = have_prev ? 0.9 * pow(C.eps / eff, 0.7 / 5.0) * pow(s.err_prev / C.eps, 0.4 / 5.0)
                           : 0.9 * pow(C.eps / eff, 0.2);
        s.h = clampd(ah * clampd(factor, 0.2, just_rej ? 2.0 : 5.0), 1e-10, fmax(hmax, 1e-10));
    } else {
        if (!C.scaled)
            factor = have_prev ? 0.9 * pow(C.eps / eff, 0.7 / order) * pow(s.err_prev / C.eps, 0.4 / order)
                               : 0.9 * pow(C.eps / eff, inv_order);
        else
            factor = have_prev ? 0.9 * pow(1.0 / eff, 0.7 / order) * pow(s.err_prev, 0.4 / order)
                               : 0.9 * pow(eff, -inv_order);
        const double mgb = fmin(1.0 + 4.0 * (5.0 / order), 5.0);
        s.h = clampd(ah * clampd(factor, 0.2, just_rej ? fmin(mgb, 2.0) : mgb), hmin, hmax);
    }
    s.err_prev = en;
    s.flags = (s.flags | kHavePrev) & ~kJustRej;
    if ((s.flags & kSegSampled) && s.t == s.seg_tf && M != kDopri5Compat && A.ctrl.h_max > 60.0 && s.h > 0.0)
        s.hcarry = s.h;  // hcarry_store (integrator.rs:206-216)
    if (A.force.ground_check) {
        double bs[6];
        baseline_state(baseline_new(s.cur), s.t - s.ct0, bs);
        const double alt = geodetic_altitude_km(bs[0] + s.y[0], bs[1] + s.y[1], bs[2] + s.y[2], A.force.earth_radius);
        if (!(alt >= kGroundAltitudeKm)) {
            traj_fail(A, s, traj, kGround);
            return;
        }
    }
    if (s.t == s.seg_tf) {
        // rectification (integrator.rs:941-979)
        const double dsq = fma(s.y[0], s.y[0], fma(s.y[1], s.y[1], s.y[2] * s.y[2]));
        if (dsq > kRebaseKm * kRebaseKm || s.seg_tf != s.tf) {
            double bs[6], e[6], ne[6];
            baseline_state(baseline_new(s.cur), s.seg_tf - s.ct0, bs);
            for (int i = 0; i < 6; ++i) e[i] = bs[i] + s.y[i];
            if (!eci_to_equinoctial(e, ne)) {
                traj_fail(A, s, traj, kRebaseFailed);
                return;
            }
            for (int i = 0; i < 6; ++i) s.cur[i] = ne[i];
            s.ct0 = s.seg_tf;
            s.flags |= kHad;
            s.phase = kNeedSegment;
        } else {
            traj_finish_with(A, s, traj, s.y);
        }
    }
}

// ------------------------------------------------- binary-eclipse coordinator
// integrate_binary_eclipse_scalar_with_rhs_inner (eclipse_coordinator.rs:
// 1228-1443), events off, as a per-row state machine over legs.  Every leg
// integrates the Encke deviation against the row's baseline (cur, ct0) with
// the eclipse side fixed, absolute max-norm error control, the end-of-step
// derivative handed forward as the next first stage and a fresh controller
// (integrate_segment_with_method, integrator.rs:404-556):
//   main    up to 5400 s; the step-size carry of the previous main leg
//   refine  the main leg's crossing step replayed with steps <= 10 s
//   proof   the old side proven up to just before the detected root
//   window  one short leg past the root; its crossing step commits the root
// A crossing found in a main / refine / proof step discards that step (its
// samples are not written); the window's crossing step is kept.

// Equinoctial elements of baseline + delta at t (the coordinator's rebase).
__device__ __forceinline__ bool ecl_rebase(const double* cur, double ct0, const double* d, double t, double* out) {
    double b[6], e[6];
    baseline_state(baseline_new(cur), t - ct0, b);
    for (int i = 0; i < 6; ++i) e[i] = b[i] + d[i];
    return eci_to_equinoctial(e, out);
}

// Open a leg at (t, y0) ending at `end` with maximum step hmax; h0 > 0 is
// the carried opening step, else span/100 (span/2 up to 60 s).
__device__ __forceinline__ void ecl_leg_start(TrajState& s, EclState& E, int32_t leg, double t, const double* y0,
                                              double end, double hmax, double h0) {
    E.leg = leg;
    s.t = t;
    for (int i = 0; i < 6; ++i) s.y[i] = y0[i];
    s.seg_tf = end;
    double hm = fabs(hmax);
    const double hmin = fmin(hm, 1e-12);
    if (hm < hmin) hm = hmin;
    s.lhmax = hm;
    const double span = fabs(end - t);
    s.h = h0 > 0.0 ? clampd(h0, hmin, hm) : clampd(span <= 60.0 ? span / 2.0 : span / 100.0, hmin, hm);
    s.err_prev = 0.0;
    s.t_comp = 0.0;
    s.flags &= kHad | kEcl;  // fresh controller, no carried first stage
    s.rejects = 0;
    s.seg_steps = 0;
    E.fch = 0.0;
    s.phase = kStepping;
}

// Main-loop top: finish at tf or open the next main leg.
template <int M>
__device__ void ecl_seg_begin(const PropArgs& A, TrajState& s, int64_t traj) {
    EclState& E = A.ecl[traj];
    const double zero[6] = {0, 0, 0, 0, 0, 0};
    if (s.ct0 == s.tf) {
        traj_finish_with(A, s, traj, zero);
        return;
    }
    if (++E.iters > kEclMaxIter) {
        traj_fail(A, s, traj, kEclSplitLimit);
        return;
    }
    const double rem = s.tf - s.ct0;
    const double end = fabs(rem) > kMaxSegmentS ? s.ct0 + kMaxSegmentS : s.tf;
    const double dtmax = A.ctrl.h_max;
    ecl_leg_start(s, E, kLegMain, s.ct0, zero, end, dtmax, dtmax > kEclHcarryMinDtMax ? s.hcarry : 0.0);
}

// Window leg from the proof point: ends at the deepest instant within the
// root budget past it (eclipse_coordinator.rs:2224-2290).
static __device__ __noinline__ void ecl_window_start(const PropArgs& A, TrajState& s, EclState& E, int64_t traj,
                                              const double* y0) {
    const EclGeo G{&A.force, s.jd0};
    double wl;
    if (int32_t e = G.deepest(E.proof_old_t, E.b2, kEclRootUncKm, &wl)) {
        traj_fail(A, s, traj, e);
        return;
    }
    if (wl < E.br_tnew) {
        traj_fail(A, s, traj, kEclNonProgress);
        return;
    }
    const double hm = fmin(fmin(A.ctrl.h_max, kEclRefineStepS), fabs(wl - E.proof_old_t));
    ecl_leg_start(s, E, kLegWindow, E.proof_old_t, y0, wl, hm, 0.0);
}

// Old-side proof leg from the transaction base (cur, ct0) to just before
// the anchor (eclipse_coordinator.rs:1995-2162); none when the base is the
// crossing itself.
static __device__ __noinline__ void ecl_proof_start(const PropArgs& A, TrajState& s, EclState& E, int64_t traj) {
    const EclGeo G{&A.force, s.jd0};
    const double base_t = s.ct0;
    const double zero[6] = {0, 0, 0, 0, 0, 0};
    double pot = base_t;
    if (E.anchor != base_t) {
        if (int32_t e = G.deepest(E.anchor, base_t, kEclOldSideMarginKm, &pot)) {
            traj_fail(A, s, traj, e);
            return;
        }
    }
    E.proof_old_t = pot;
    s.s_idx = E.idx_base;  // a restarted proof rewrites its samples
    if (!ecl_envelope(baseline_new(s.cur), base_t, zero, base_t)) {
        traj_fail(A, s, traj, kEclEnvelope);
        return;
    }
    if (pot == base_t) {
        ecl_window_start(A, s, E, traj, zero);
        return;
    }
    const double hm = fmin(fmin(A.ctrl.h_max, kEclRefineStepS), fabs(pot - base_t));
    ecl_leg_start(s, E, kLegProof, base_t, zero, pot, hm, 0.0);
}

// A crossing found in the accepted step [s.t, tn] of the current leg.
static __device__ __noinline__ void ecl_crossing(const PropArgs& A, TrajState& s, EclState& E, int64_t traj,
                                          const EclBracket& br, double tn, const double* ynext) {
    const double dtmax = A.ctrl.h_max;
    const double zero[6] = {0, 0, 0, 0, 0, 0};
    if (E.leg == kLegMain) {
        // resolve_eclipse_split (1453-1619): replay the step from its start
        if (dtmax > kEclHcarryMinDtMax && E.fch > 0.0) s.hcarry = E.fch;
        const double a = s.t, b = tn;
        double re[6];
        if (!ecl_rebase(s.cur, s.ct0, s.y, a, re)) return traj_fail(A, s, traj, kRebaseFailed);
        if (!isfinite(a) || !isfinite(b) || a == b || br.old_side == br.new_side)
            return traj_fail(A, s, traj, kEclBracket);
        for (int i = 0; i < 6; ++i) s.cur[i] = re[i];
        s.ct0 = a;
        if (!ecl_envelope(baseline_new(s.cur), a, zero, a)) return traj_fail(A, s, traj, kEclEnvelope);
        E.a = a;
        E.b = b;
        E.br_old = br.old_side;
        E.br_new = br.new_side;
        ecl_leg_start(s, E, kLegRefine, a, zero, b, fmin(dtmax, kEclRefineStepS), 0.0);
        return;
    }
    if (E.leg == kLegRefine) {
        // refine_eclipse_bracket's checks (1621-1738), rebase at the fine
        // step's start, then the root transaction (2164-2370)
        if (br.old_side != E.br_old || br.new_side == E.br_old || !isfinite(br.bound) ||
            !(br.bound >= 0.0 && br.bound <= kEclMaxSepKm))
            return traj_fail(A, s, traj, kEclBracket);
        if (!(E.a <= s.t && s.t < tn && tn <= E.b)) return traj_fail(A, s, traj, kEclNonProgress);
        double re[6];
        if (!ecl_rebase(s.cur, s.ct0, s.y, s.t, re)) return traj_fail(A, s, traj, kRebaseFailed);
        for (int i = 0; i < 6; ++i) s.cur[i] = re[i];
        s.ct0 = s.t;
        E.b2 = tn;
        E.br_told = br.t_old;
        E.br_tnew = br.t_new;
        E.br_old = br.old_side;
        E.br_new = br.new_side;
        E.anchor = br.t_old;
        E.restarts = kEclProofRestarts;
        E.idx_base = s.s_idx;
        ecl_proof_start(A, s, E, traj);
        return;
    }
    if (E.leg == kLegProof) {
        // the proof leg found the crossing earlier than its anchor: restart
        // from that better-resolved anchor (2076-2162)
        const double ft = br.t_old;
        if (E.restarts == 0 || !isfinite(ft) || !(ft < E.anchor) || br.old_side != E.br_old)
            return traj_fail(A, s, traj, kEclBracket);
        --E.restarts;
        E.anchor = ft;
        ecl_proof_start(A, s, E, traj);
        return;
    }
    // window: validate_eclipse_root_commit (1879-1926), rebase_after_eclipse_root (1928-1993)
    const double ev = tn;
    if (br.old_side != E.br_old || br.new_side != E.br_new) return traj_fail(A, s, traj, kEclBracket);
    const Baseline bb = baseline_new(s.cur);
    if (!ecl_envelope(bb, s.ct0, ynext, ev)) return traj_fail(A, s, traj, kEclEnvelope);
    const EclGeo G{&A.force, s.jd0};
    int cs;
    double cm, unc;
    if (int32_t e = ecl_side_at(G, bb, s.ct0, ynext, ev, &cs, &cm)) return traj_fail(A, s, traj, e);
    if (int32_t e = G.replay_unc(E.proof_old_t, ev, &unc)) return traj_fail(A, s, traj, e);
    if (cs != br.new_side || unc > kEclRootUncKm) return traj_fail(A, s, traj, kEclBracket);
    if (!isfinite(ev) || ev == s.t || (E.have_root && ev <= E.root_t)) return traj_fail(A, s, traj, kEclChatter);
    if (++E.splits > kEclMaxSplits) return traj_fail(A, s, traj, kEclSplitLimit);
    double b[6], eci[6], re[6];
    baseline_state(bb, ev - s.ct0, b);
    for (int i = 0; i < 6; ++i) eci[i] = b[i] + ynext[i];
    if (!eci_to_equinoctial(eci, re)) return traj_fail(A, s, traj, kRebaseFailed);
    for (int i = 0; i < 6; ++i) s.cur[i] = re[i];
    s.ct0 = ev;
    s.side = br.new_side;
    double rb[6], terr;
    baseline_state(baseline_new(s.cur), 0.0, rb);
    if (!ecl_outward(dist3(eci, rb), &terr)) return traj_fail(A, s, traj, kEclGeometry);
    if (terr > kEclMaxSepKm) return traj_fail(A, s, traj, kEclBracket);
    E.have_root = 1;
    E.root_t = ev;
    E.root_err = terr;
    s.phase = kNeedSegment;
}

// The current leg reached its end without a crossing.
static __device__ __noinline__ void ecl_leg_done(const PropArgs& A, TrajState& s, EclState& E, int64_t traj) {
    if (E.leg == kLegMain || E.leg == kLegRefine) {
        // complete_non_eclipse_segment (2372-2583)
        if (E.leg == kLegMain && A.ctrl.h_max > kEclHcarryMinDtMax && E.fch > 0.0) s.hcarry = E.fch;
        if (s.seg_tf == s.tf) {
            traj_finish_with(A, s, traj, s.y);
            return;
        }
        double re[6];
        if (!ecl_rebase(s.cur, s.ct0, s.y, s.seg_tf, re)) return traj_fail(A, s, traj, kRebaseFailed);
        for (int i = 0; i < 6; ++i) s.cur[i] = re[i];
        s.ct0 = s.seg_tf;
        E.have_root = 0;
        s.phase = kNeedSegment;
        return;
    }
    if (E.leg == kLegProof) {
        // proven_old_side_delta (2028-2048), then the window leg
        const Baseline bb = baseline_new(s.cur);
        if (!ecl_envelope(bb, s.ct0, s.y, s.t)) return traj_fail(A, s, traj, kEclEnvelope);
        const EclGeo G{&A.force, s.jd0};
        int ps;
        double pm;
        if (int32_t e = ecl_side_at(G, bb, s.ct0, s.y, s.t, &ps, &pm)) return traj_fail(A, s, traj, e);
        if (ps != E.br_old) return traj_fail(A, s, traj, kEclBracket);
        double y0[6];
        for (int i = 0; i < 6; ++i) y0[i] = s.y[i];
        ecl_window_start(A, s, E, traj, y0);
        return;
    }
    traj_fail(A, s, traj, kEclBracket);  // a window leg without its crossing
}

// The scan an accepted SRP step asks for.
struct EclScanReq {
    EclPath H;
    double from, t1;
    EclPoint start;  // the point at `from`
};

// Accepted step of an SRP row, up to its crossing scan: the time update and
// the handler's checks.  False when the row failed (its status is written).
template <int M>
__device__ __noinline__ bool ecl_accept_pre(const PropArgs& A, TrajState& s, int64_t traj, const double* ynext,
                                            const double* dy_prev, const double* dy_next, double* tn_out,
                                            EclScanReq* req) {
    double tn;
    if (s.flags & kLands) {
        tn = s.seg_tf;
    } else {
        const double ky = s.hs - s.t_comp;
        const double nx = s.t + ky;
        s.t_comp = (nx - s.t) - ky;
        tn = nx;
    }
    if (!isfinite(tn)) {
        traj_fail(A, s, traj, kNonFinite);
        return false;
    }
    ++s.seg_steps;
    ++s.steps;
    s.rejects = 0;
    const EclGeo G{&A.force, s.jd0};
    if (int32_t e = ecl_step_pre(G, baseline_new(s.cur), s.ct0, s.side, A.ecl[traj], s.t, s.y, dy_prev, tn, ynext,
                                 dy_next, &req->H, &req->from, &req->start)) {
        traj_fail(A, s, traj, e);
        return false;
    }
    req->t1 = tn;
    *tn_out = tn;
    return true;
}

// The rest of the accepted step after its scan: samples, the carried first
// stage, the PI controller, a crossing's leg change or the leg's end.
template <int M>
__device__ __noinline__ void ecl_accept_post(const PropArgs& A, TrajState& s, int64_t traj, double tn,
                                             const double* ynext, const double* dy_prev, const double* dy_next,
                                             double en, int32_t scan_err, bool found, const EclBracket& br) {
    using T = Tab<M>;
    const CtrlParams& C = A.ctrl;
    EclState& E = A.ecl[traj];
    if (scan_err) return traj_fail(A, s, traj, scan_err);
    if (found && br.old_side != s.side) return traj_fail(A, s, traj, kEclChatter);
    const bool keep = !found || E.leg == kLegWindow;
    if (keep && sampled_mode(A)) emit_samples(A, s, traj, tn, ynext, dy_prev, dy_next);
    if (keep && A.force.ground_check) {
        double bs[6];
        baseline_state(baseline_new(s.cur), tn - s.ct0, bs);
        const double alt = geodetic_altitude_km(bs[0] + ynext[0], bs[1] + ynext[1], bs[2] + ynext[2],
                                                A.force.earth_radius);
        if (!(alt >= kGroundAltitudeKm)) return traj_fail(A, s, traj, kGround);
    }
    if (found) {
        ecl_crossing(A, s, E, traj, br, tn, ynext);
        return;
    }
    for (int i = 0; i < 6; ++i) s.k1c[i] = dy_next[i];
    s.flags |= kHaveK1;
    const double ah = fabs(s.hs);
    s.t = tn;
    for (int i = 0; i < 6; ++i) s.y[i] = ynext[i];
    // pi_controller_accept! (solver.rs:445-503), absolute control
    const double order = (double)T::ORDER_ERR + 1.0;
    const double eff = en > 0.0 ? en : C.eps * 0.1;
    const bool have_prev = (s.flags & kHavePrev) && s.err_prev > 0.0;
    const double factor = have_prev ? 0.9 * pow(C.eps / eff, 0.7 / order) * pow(s.err_prev / C.eps, 0.4 / order)
                                    : 0.9 * pow(C.eps / eff, 1.0 / order);
    const double mgb = fmin(1.0 + 4.0 * (5.0 / order), 5.0);
    s.h = clampd(ah * clampd(factor, 0.2, (s.flags & kJustRej) ? fmin(mgb, 2.0) : mgb), C.h_min, s.lhmax);
    E.fch = s.h;
    s.err_prev = en;
    s.flags = (s.flags | kHavePrev) & ~kJustRej;
    if (s.t == s.seg_tf) ecl_leg_done(A, s, E, traj);
}

// Accepted step of an SRP row scanned by its own thread (the persistent
// engine; the stage-synchronous engine scans warp-cooperatively).
template <int M>
__device__ __noinline__ void ecl_accept(const PropArgs& A, TrajState& s, int64_t traj, const double* ynext,
                                        const double* dy_prev, const double* dy_next, double en) {
    double tn;
    EclScanReq req;
    if (!ecl_accept_pre<M>(A, s, traj, ynext, dy_prev, dy_next, &tn, &req)) return;
    const EclGeo G{&A.force, s.jd0};
    bool found = false;
    EclBracket br;
    const int32_t e = ecl_first_crossing(G, req.H, req.from, req.t1, &found, &br, kEclMaxSplits, &req.start);
    ecl_accept_post<M>(A, s, traj, tn, ynext, dy_prev, dy_next, en, e, found, br);
}

}  // namespace bqp
