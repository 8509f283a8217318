// Stage-synchronous propagation engine.
//
// The persistent kernel (propagate.cu) runs the whole force model and the
// controller inside one thread per trajectory; at 70x70 + JB2008 that kernel
// is large, register-bound (255 registers, 8 warps per SM) and stalls on
// instruction fetch.  Here every RK stage of every active trajectory is one
// pass over three specialised kernels, and one controller kernel closes the
// attempt:
//
//   pl_prep<M>(s)   finish stage s-1, form y_s = y + h sum a_sj k_j, the Encke
//                   baseline (Kepler solve), Earth rotation, Sun/Moon third body
//                   and Battin's term                       (latency / SFU bound)
//   pl_gravity      normalised column recursion, table in shared memory,
//                   one trajectory per thread               (FP64-FMA bound)
//   pl_drag         JB2008 density and co-rotating drag     (transcendental bound)
//   pl_control<M>   finish the last stage, error norm, accept / reject, samples,
//                   rectification, next attempt; compacts the active list
//
// Stage data are indexed by the trajectory's slot in the active list, so the
// force kernels stream contiguous arrays; the active list shrinks as
// trajectories finish.  The attempt sequence is captured once as a CUDA graph
// and replayed; the host reads the active count between replays.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <vector>

#include "kernels.cuh"
#include "launch.h"
#include "traj.cuh"

namespace bqp {

namespace {

constexpr int kBlock = 256;

// Drag lanes per state above and below ~510 km (the lanes share the sweep
// series and the intervals walked exactly), and the drag kernel's minimum
// resident CTAs per SM, which sets its register budget (3: 80 registers, a
// few hundred bytes spilled).  Measured on 65,536 LEO states at 70x70: one
// lane above 510 km and four below, both lists in one launch at 3 CTAs per
// SM, fit every state of a stage in one wave; that took the drag kernels
// from 1,023 ms to 701 ms per 5,400 s segment.
#ifndef BQP_DRAG_LANES_HIGH
#define BQP_DRAG_LANES_HIGH 1
#endif
#ifndef BQP_DRAG_LANES_LOW
#define BQP_DRAG_LANES_LOW 4
#endif
#ifndef BQP_DRAG_MIN_BLOCKS
#define BQP_DRAG_MIN_BLOCKS 3
#endif
// stage derivative buffers per row: the most stages of any tableau (Vern9's
// 16) plus the dense-output stage of the sampled non-FSAL path
constexpr int kStageBufs = Tab<kVern9>::S + 1;

__device__ __forceinline__ double* K(const PipeBufs& P, int st, int i) { return P.k + ((size_t)st * 6 + i) * P.cap; }

// Append `traj` to the next active list (warp-aggregated atomic).
__device__ __forceinline__ void append_active(int32_t* list, int32_t* count, int32_t traj, bool keep) {
    const unsigned mask = __ballot_sync(0xffffffffu, keep);
    if (!keep) return;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(count, __popc(mask));
    base = __shfl_sync(mask, base, leader);
    const int rank = __popc(mask & ((1u << lane) - 1u));
    list[base + rank] = traj;
}

// Sum of the stage-`st` force terms into K(st, 3..5).
__device__ __forceinline__ void finish_stage(const PipeBufs& P, int st, int slot) {
    const double gx = P.agrav[slot], gy = P.agrav[P.cap + slot], gz = P.agrav[2 * P.cap + slot];
    if (P.iau) {
        double r[9], g[3];
        const double gi[3] = {gx, gy, gz};
        for (int e = 0; e < 9; ++e) r[e] = P.fr[(size_t)e * P.cap + slot];
        ft::to_gcrs(r, gi, g);
        for (int i = 0; i < 3; ++i)
            K(P, st, 3 + i)[slot] = g[i] + P.adrag[(size_t)i * P.cap + slot] + P.part[(size_t)i * P.cap + slot];
        return;
    }
    const double s = P.sc[slot], c = P.sc[P.cap + slot];
    K(P, st, 3)[slot] = fma(c, gx, -s * gy) + P.adrag[slot] + P.part[slot];
    K(P, st, 4)[slot] = fma(s, gx, c * gy) + P.adrag[P.cap + slot] + P.part[P.cap + slot];
    K(P, st, 5)[slot] = gz + P.adrag[2 * P.cap + slot] + P.part[2 * P.cap + slot];
}

// An ECI vector of slot `slot` in the Earth-fixed frame of its stage.
__device__ __forceinline__ void slot_to_itrs(const PipeBufs& P, int slot, const double* v, double* o) {
    if (P.iau) {
        double r[9];
        for (int e = 0; e < 9; ++e) r[e] = P.fr[(size_t)e * P.cap + slot];
        ft::to_itrs(r, v, o);
    } else {
        const double s = P.sc[slot], c = P.sc[P.cap + slot];
        o[0] = fma(c, v[0], s * v[1]);
        o[1] = fma(-s, v[0], c * v[1]);
        o[2] = v[2];
    }
}

}  // namespace

// --------------------------------------------------------------------- init
template <int M>
__global__ void __launch_bounds__(kBlock) pl_init(PropArgs A, PipeBufs P) {
    const int64_t traj = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool keep = false;
    if (traj < A.n) {
        TrajState s;
        traj_begin(A, s, traj);
        if (s.phase == kNeedSegment) seg_begin<M>(A, s, traj);
        if (s.phase == kStepping) {
            const int32_t f = attempt_begin<M>(A, s, false);
            if (f >= 0) traj_fail(A, s, traj, f);
            else keep = true;
        }
        P.st[traj] = s;
    }
    append_active(P.idx[0], &P.count[0], (int32_t)traj, keep);
}

// --------------------------------------------------------------------- prep
// Stage `st` of the current attempt.  st == S is the dense-output stage of
// the sampled non-FSAL path: f(t_next, y_next) evaluated before the
// controller decides (the reference evaluates it after an accept).
template <int M>
__global__ void __launch_bounds__(kBlock) pl_prep(PropArgs A, PipeBufs P, int cur, int st) {
    using T = Tab<M>;
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (st == 0 && blockIdx.x == 0 && threadIdx.x == 0) P.count[cur ^ 1] = 0;
    if (slot >= P.count[cur]) return;
    const int32_t traj = P.idx[cur][slot];
    const TrajState& s = P.st[traj];
    if (st == 0) {
        P.bad[slot] = 0;
        if (s.flags & kHaveK1) {
            for (int i = 0; i < 6; ++i) K(P, 0, i)[slot] = s.k1c[i];
            P.skip[slot] = 1;
            return;
        }
    } else if (!(st == 1 && P.skip[slot])) {
        finish_stage(P, st - 1, slot);
    }
    P.skip[slot] = 0;
    // stage state
    double yt[6];
    for (int i = 0; i < 6; ++i) yt[i] = s.y[i];
    double ts;
    if (st < T::S) {
#pragma unroll 1
        for (int j = 0; j < st; ++j) {
            const double a = s.hs * T::a(st, j);
            if (a != 0.0)
                for (int i = 0; i < 6; ++i) yt[i] = fma(K(P, j, i)[slot], a, yt[i]);
        }
        ts = s.t + T::c(st) * s.hs;
    } else {
        // y_next exactly as rk_combine forms it
#pragma unroll 1
        for (int j = 0; j < T::S; ++j) {
            const double b = s.hs * T::b(j);
            if (b != 0.0)
                for (int i = 0; i < 6; ++i) yt[i] = fma(K(P, j, i)[slot], b, yt[i]);
        }
        ts = next_time(s);
    }
    double rs[6];
    baseline_state(baseline_new(s.cur), ts - s.ct0, rs);
    double sp[6];
    for (int i = 0; i < 6; ++i) {
        sp[i] = rs[i] + yt[i];
        P.sp[(size_t)i * P.cap + slot] = sp[i];
    }
    for (int i = 0; i < 3; ++i) K(P, st, i)[slot] = yt[3 + i];
    const double jd = utc_jd_at(s.jd0, ts);
    const ForceParams& fp = A.force;
    if (P.iau) {
        // the IAU 2006/2000A rotation of the stage's instant (rhs.rs:3113-3174)
        ft::FrameRot F;
        if ((fp.gravity_on || fp.drag) && !frame_rot(fp.frame, s.tai0 + ts, F)) {
            P.bad[slot] = 3;
            for (int e = 0; e < 9; ++e) F.r[e] = NAN;
            F.w[0] = F.w[1] = F.w[2] = NAN;
        } else if (!(fp.gravity_on || fp.drag)) {
            for (int e = 0; e < 9; ++e) F.r[e] = (e % 4 == 0) ? 1.0 : 0.0;
            F.w[0] = F.w[1] = F.w[2] = 0.0;
        }
        for (int e = 0; e < 9; ++e) P.fr[(size_t)e * P.cap + slot] = F.r[e];
        for (int e = 0; e < 3; ++e) P.fr[(size_t)(9 + e) * P.cap + slot] = F.w[e];
    } else {
        double sn = 0.0, cs = 1.0;
        if (fp.gravity_on || fp.drag) sincos(gmst_rad(jd), &sn, &cs);
        P.sc[slot] = sn;
        P.sc[P.cap + slot] = cs;
    }
    double acc[3] = {0.0, 0.0, 0.0};
    double sun[3];
    const bool need_sun = fp.sun || (fp.drag && s.cd != 0.0 && s.am != 0.0) || s.side >= 0;
    if (need_sun) sun_at(fp.eph_sun, jd, sun);
    if (s.side >= 0) srp_accel(sp, sun, fp.p_sun, fp.cr, s.am, s.side, acc);  // on the leg's fixed side
    if (fp.sun) third_body(sp, sun, fp.mu_sun, acc);
    if (fp.moon) {
        double moon[3];
        moon_at(fp.eph_moon, jd, moon);
        third_body(sp, moon, fp.mu_moon, acc);
    }
    const double r2 = fma(sp[0], sp[0], fma(sp[1], sp[1], sp[2] * sp[2]));
    battin(rs, yt, r2, sqrt(r2), acc);
    for (int i = 0; i < 3; ++i) P.part[(size_t)i * P.cap + slot] = acc[i];
    if (fp.drag) {
        for (int i = 0; i < 3; ++i) P.sun[(size_t)i * P.cap + slot] = sun[i];
        P.jd[slot] = jd;
        P.amcd[slot] = s.am;
        P.amcd[P.cap + slot] = s.cd;
        // drag work list: states above ~510 km take the sweep fits (cheap),
        // the rest walk the quadrature; homogeneous warps in each list
        const int cls = sqrt(r2) - fp.earth_radius >= 510.0 ? 0 : 1;
        const unsigned m = __activemask();
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const unsigned mm = __ballot_sync(m, cls == c);
            if (cls == c) {
                const int lane = threadIdx.x & 31;
                const int leader = __ffs(mm) - 1;
                int base = 0;
                if (lane == leader) base = atomicAdd(&P.dcount[c], __popc(mm));
                base = __shfl_sync(mm, base, leader);
                P.dlist[c][base + __popc(mm & ((1u << lane) - 1u))] = slot;
            }
        }
    } else {
        for (int i = 0; i < 3; ++i) P.adrag[(size_t)i * P.cap + slot] = 0.0;
    }
    if (!fp.gravity_on)
        for (int i = 0; i < 3; ++i) P.agrav[(size_t)i * P.cap + slot] = 0.0;
}

// ------------------------------------------------------------------ gravity
// Persistent over slots: one CTA per SM stages the field table once; the
// CTA's contiguous slot range is walked NT slots per thread.
// `out` receives the field; with `list` set the rows are the slots
// list[0 .. *list_count) instead of the active slots 0 .. count.
template <int NT>
__global__ void __launch_bounds__(256, 1) pl_gravity(GravTable T, int parts_max, PipeBufs P, int cur, double* out,
                                                     const int32_t* list, const int32_t* list_count) {
    const int count = list ? *list_count : P.count[cur];
    const int per_block = (count + gridDim.x - 1) / gridDim.x;
    const int b0 = blockIdx.x * per_block;
    const int b1 = min(count, b0 + per_block);
    if (b0 >= b1) return;  // uniform across the CTA
    auto load = [&](int row, double& x, double& y, double& z) -> bool {
        const int sl = list ? list[row] : row;
        if (P.skip[sl]) return false;
        const double e[3] = {P.sp[sl], P.sp[P.cap + sl], P.sp[2 * P.cap + sl]};
        double q[3];
        slot_to_itrs(P, sl, e, q);
        const double r2 = fma(q[0], q[0], fma(q[1], q[1], q[2] * q[2]));
        if (!(isfinite(r2) && r2 > 0.0)) {
            if (!P.bad[sl]) P.bad[sl] = 1;
            out[sl] = out[P.cap + sl] = out[2 * P.cap + sl] = NAN;
            return false;
        }
        x = q[0];
        y = q[1];
        z = q[2];
        return true;
    };
    auto store = [&](int row, const double* a, double, double, double) {
        const int sl = list ? list[row] : row;
        out[sl] = a[0];
        out[P.cap + sl] = a[1];
        out[2 * P.cap + sl] = a[2];
    };
    auto lost = [&](int row) {
        const int sl = list ? list[row] : row;
        P.bad[sl] = 2;
        out[sl] = out[P.cap + sl] = out[2 * P.cap + sl] = NAN;
    };
    gravity_cta<NT>(T, parts_max, per_block, b0, b1, load, store, lost);
}

// Earth-fixed positions of the stage's active slots, [slot][3] (the
// surrogate's input)
__global__ void __launch_bounds__(kBlock) pl_earth_fixed(PipeBufs P, int cur) {
    const int sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= P.count[cur]) return;
    const double e[3] = {P.sp[sl], P.sp[P.cap + sl], P.sp[2 * P.cap + sl]};
    slot_to_itrs(P, sl, e, P.ef + 3 * (size_t)sl);
}

// ------------------------------------------------------- surrogate check
// Per step, at its first stage: the network's field (agrav) against the
// exact one (agx), both without the central term.  A row off by more than
// `thr` of the whole exact field's magnitude (central term included) takes
// the exact field now and, through the slot list, at the step's later
// stages.  A row whose first stage was carried over (a retried step, or the
// FSAL stage of the step before) keeps the verdict under which that stage
// was evaluated.
__global__ void __launch_bounds__(kBlock) pl_sur_check(PipeBufs P, int cur, double thr) {
    const int sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= P.count[cur]) return;
    const int32_t traj = P.idx[cur][sl];
    if (!P.skip[sl]) {
        const double* q = P.ef + 3 * (size_t)sl;  // Earth-fixed position
        const double r2 = fma(q[0], q[0], fma(q[1], q[1], q[2] * q[2]));
        const double kc = -kMu / (r2 * sqrt(r2));
        double d2 = 0.0, a2 = 0.0;
        for (int k = 0; k < 3; ++k) {
            const size_t o = (size_t)k * P.cap + sl;
            const double d = P.agrav[o] - P.agx[o];
            const double a = fma(kc, q[k], P.agx[o]);
            d2 = fma(d, d, d2);
            a2 = fma(a, a, a2);
        }
        const bool fall = !(d2 <= thr * thr * a2);  // NaN falls back too
        P.fall[traj] = fall ? 1 : 0;
        if (fall)
            for (int k = 0; k < 3; ++k) P.agrav[(size_t)k * P.cap + sl] = P.agx[(size_t)k * P.cap + sl];
    }
    if (P.fall[traj]) P.flist[atomicAdd(P.fcount, 1)] = sl;
}

// --------------------------------------------------------------------- drag
// One state per group of L lanes (jb::density_group): the JB2008 model is the
// longest serial chain of the force call, and the kernel is bound by that
// latency, not by throughput.  Both drag lists go in one launch (blocks
// [0, nb_hi) take list 0 with LH lanes per state, the rest list 1 with LL),
// so that a stage's states are resident together in as few waves as the
// register budget allows.
template <int L, bool kCoarse = false>
__device__ __forceinline__ void drag_rows(const ForceParams& fp, const PipeBufs& P, int list, int block) {
    const int gt = block * blockDim.x + threadIdx.x;
    const int item = gt / L;
    const int q = gt % L;
    const unsigned gmask = ((1u << L) - 1u) << ((threadIdx.x & 31) & ~(L - 1));
    if (item >= P.dcount[list]) return;  // uniform across the group
    const int slot = P.dlist[list][item];
    double sp[6];
    for (int i = 0; i < 6; ++i) sp[i] = P.sp[(size_t)i * P.cap + slot];
    const double am = P.amcd[slot], cd = P.amcd[P.cap + slot];
    double a[3] = {0.0, 0.0, 0.0};
    if (cd != 0.0 && am != 0.0) {
        // JB2008 adapter (rhs.rs:3551-3776), as Encke::density_at
        const double sun[3] = {P.sun[slot], P.sun[P.cap + slot], P.sun[2 * P.cap + slot]};
        double pi[3], si[3];
        slot_to_itrs(P, slot, sp, pi);
        slot_to_itrs(P, slot, sun, si);
        const double sun_r = sqrt(fma(si[0], si[0], fma(si[1], si[1], si[2] * si[2])));
        const double sat_r = sqrt(fma(pi[0], pi[0], fma(pi[1], pi[1], pi[2] * pi[2])));
        double rho;
        if ((sat_r - fp.earth_radius) * 1000.0 > 2500.0e3) {
            rho = 1.0e-19;
        } else {
            const double alt_m = geodetic_altitude_km(pi[0], pi[1], pi[2], fp.earth_radius) * 1000.0;
            const double dec = asin(fmin(1.0, fmax(-1.0, si[2] / sun_r)));
            const double ha = atan2(fma(pi[1], si[0], -(pi[0] * si[1])), fma(pi[0], si[0], pi[1] * si[1]));
            const double lat = asin(fmin(1.0, fmax(-1.0, pi[2] / sat_r)));
            jb::Drivers dr = fp.drivers;
            // fixed-node fits from constant memory (fp.fit holds the same numbers);
            // no drivers at this instant -> NaN density (rhs.rs:3560-3571), the
            // same verdict on every lane of the group
            if (fp.dtab.n_solar > 0 && !jb::lookup_drivers(fp.dtab, P.jd[slot], &dr))
                rho = NAN;
            else if (kCoarse && fp.drag_fp32)
                rho = jb::density_coarse_r<float>(P.jd[slot] - 2400000.5, dec, ha, lat, alt_m, dr, fp.atm_model);
            else if (kCoarse)
                rho = jb::density_coarse(P.jd[slot] - 2400000.5, dec, ha, lat, alt_m, dr, fp.atm_model);
            else
                rho = jb::density_group<L>(P.jd[slot] - 2400000.5, dec, ha, lat, alt_m, dr, q, gmask,
                                           fp.fit != nullptr, fp.fit2);
            if (!(rho > 0.0) || !isfinite(rho)) rho = NAN;
            else if (alt_m > 2500.0e3) rho = fmin(rho, 1.0e-19);
        }
        if (isnan(rho)) {
            a[0] = a[1] = a[2] = NAN;
        } else if (rho > 0.0) {
            double vr0, vr1, vr2;
            if (P.iau) {
                // atmosphere co-rotating with the resolved frame (rhs.rs:1134-1139)
                double w[3];
                for (int e = 0; e < 3; ++e) w[e] = P.fr[(size_t)(9 + e) * P.cap + slot];
                vr0 = (sp[3] - (w[1] * sp[2] - w[2] * sp[1])) * 1000.0;
                vr1 = (sp[4] - (w[2] * sp[0] - w[0] * sp[2])) * 1000.0;
                vr2 = (sp[5] - (w[0] * sp[1] - w[1] * sp[0])) * 1000.0;
            } else {
                const double w = fp.omega;
                vr0 = (sp[3] + w * sp[1]) * 1000.0;
                vr1 = (sp[4] - w * sp[0]) * 1000.0;
                vr2 = sp[5] * 1000.0;
            }
            const double v2 = fma(vr0, vr0, fma(vr1, vr1, vr2 * vr2));
            if (v2 != 0.0) {
                const double k = -0.5 * cd * am * rho * sqrt(v2) * 1e-3;
                a[0] = k * vr0;
                a[1] = k * vr1;
                a[2] = k * vr2;
            }
        }
    }
    if (q == 0)
        for (int i = 0; i < 3; ++i) P.adrag[(size_t)i * P.cap + slot] = a[i];
}

template <int LH, int LL>
__global__ void __launch_bounds__(kBlock, BQP_DRAG_MIN_BLOCKS) pl_drag(ForceParams fp, PipeBufs P, int nb_hi) {
    if ((int)blockIdx.x < nb_hi) drag_rows<LH>(fp, P, 0, blockIdx.x);
    else drag_rows<LL>(fp, P, 1, blockIdx.x - nb_hi);
}

// The coarse profiles (atm_model 5-7): a short chain per state, one lane
// each, both altitude lists in one launch.
__global__ void __launch_bounds__(kBlock) pl_drag_coarse(ForceParams fp, PipeBufs P, int nb_hi) {
    if ((int)blockIdx.x < nb_hi) drag_rows<1, true>(fp, P, 0, blockIdx.x);
    else drag_rows<1, true>(fp, P, 1, blockIdx.x - nb_hi);
}

// ------------------------------------------------------------------ control
// Splits a row's own thread may take on its crossing scan before the warp
// takes it over.
#ifndef BQP_ECL_SOLO_SPLITS
#define BQP_ECL_SOLO_SPLITS 4
#endif
constexpr int64_t kEclSoloSplits = BQP_ECL_SOLO_SPLITS;

template <int M>
__global__ void __launch_bounds__(kBlock) pl_control(PropArgs A, PipeBufs P, int cur, int dense,
                                                      int timed_out) {
    using T = Tab<M>;
    // per warp: the store of the cooperative eclipse scan (SRP rows)
    __shared__ EclWarpStore ecl_ws[kBlock / 32];
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const int count = P.count[cur];
    if (slot - lane >= count) return;  // the whole warp is idle
    const bool active = slot < count;
    bool keep = false;
    int32_t traj = 0;
    TrajState s;
    bool scan = false;  // an accepted SRP step waiting for its crossing scan
    EclScanReq req;
    double tn = 0.0, en = 0.0, ynext[6], k0[6], dyn[6];
    if (active) {
        traj = P.idx[cur][slot];
        s = P.st[traj];
        const int last = dense ? T::S : T::S - 1;
        if (!(last == 1 && P.skip[slot])) finish_stage(P, last, slot);
        // stage derivatives of this attempt
        const int evaluated = T::S - ((s.flags & kHaveK1) ? 1 : 0);
        s.evals += evaluated;
        double err[6], err3[6];
        rk_combine<M>(s, [&](int st, int i) { return K(P, st, i)[slot]; }, ynext, err, err3);
        for (int i = 0; i < 6; ++i) k0[i] = K(P, 0, i)[slot];
        int32_t code = -1;
        const int32_t d = attempt_decide<M>(A, s, k0, ynext, err, err3, &en, &code);
        if (P.bad[slot]) {
            traj_fail(A, s, traj, P.bad[slot] == 2 ? kWatchdog : P.bad[slot] == 3 ? kFrameTime : kGravityRadius);
        } else if (d == kFail) {
            traj_fail(A, s, traj, code);
        } else if (d == kAccept) {
            const double* dy_next = nullptr;
            if (T::FSAL) {
                for (int i = 0; i < 6; ++i) dyn[i] = K(P, T::S - 1, i)[slot];
                dy_next = dyn;
            } else if (dense && (s.flags & (kSegSampled | kEcl))) {
                for (int i = 0; i < 6; ++i) dyn[i] = K(P, T::S, i)[slot];
                dy_next = dyn;
                ++s.evals;  // counted on accept only, as the reference evaluates it
            }
            if (M != kDopri5Compat && (s.flags & kEcl)) {
                // most steps are certified free of crossings after a few
                // splits; the rest go to the warp
                if (ecl_accept_pre<M>(A, s, traj, ynext, k0, dyn, &tn, &req)) {
                    const EclGeo G{&A.force, s.jd0};
                    bool found = false;
                    EclBracket br{};
                    const int32_t e =
                        ecl_first_crossing(G, req.H, req.from, req.t1, &found, &br, kEclSoloSplits, &req.start);
                    if (e == kEclDefer) scan = true;
                    else ecl_accept_post<M>(A, s, traj, tn, ynext, k0, dyn, en, e, found, br);
                }
            } else
                attempt_accept<M>(A, s, traj, ynext, k0, dy_next, en);
        }
    }
    if (A.force.srp) {
        // the warp scans each waiting row's step together, one row at a time
        int32_t scan_err = kOk;
        bool scan_found = false;
        EclBracket scan_br{};
        unsigned want = __ballot_sync(0xffffffffu, scan);
        while (want) {
            const int leader = __ffs(want) - 1;
            want &= want - 1;
            EclPath H;
            for (int i = 0; i < 3; ++i) {
                H.p0[i] = __shfl_sync(0xffffffffu, req.H.p0[i], leader);
                H.v0[i] = __shfl_sync(0xffffffffu, req.H.v0[i], leader);
                H.p1[i] = __shfl_sync(0xffffffffu, req.H.p1[i], leader);
                H.v1[i] = __shfl_sync(0xffffffffu, req.H.v1[i], leader);
            }
            H.t0 = __shfl_sync(0xffffffffu, req.H.t0, leader);
            H.t1 = __shfl_sync(0xffffffffu, req.H.t1, leader);
            const double from = __shfl_sync(0xffffffffu, req.from, leader);
            const double t1 = __shfl_sync(0xffffffffu, req.t1, leader);
            const double jd0 = __shfl_sync(0xffffffffu, s.jd0, leader);
            EclPoint q;
            q.t = __shfl_sync(0xffffffffu, req.start.t, leader);
            for (int i = 0; i < 3; ++i) {
                q.p[i] = __shfl_sync(0xffffffffu, req.start.p[i], leader);
                q.v[i] = __shfl_sync(0xffffffffu, req.start.v[i], leader);
            }
            q.side = __shfl_sync(0xffffffffu, req.start.side, leader);
            q.margin = __shfl_sync(0xffffffffu, req.start.margin, leader);
            const EclGeo G{&A.force, jd0};
            bool found = false;
            EclBracket br{};
            const int32_t e = ecl_first_crossing_warp(G, H, from, t1, ecl_ws[threadIdx.x >> 5], &found, &br, &q);
            if (lane == leader) {
                scan_err = e;
                scan_found = found;
                scan_br = br;
            }
        }
        if (scan) ecl_accept_post<M>(A, s, traj, tn, ynext, k0, dyn, en, scan_err, scan_found, scan_br);
    }
    if (active) {
        if (s.phase == kNeedSegment) seg_begin<M>(A, s, traj);
        if (s.phase == kStepping) {
            const int32_t f = attempt_begin<M>(A, s, timed_out != 0);
            if (f >= 0) traj_fail(A, s, traj, f);
            else keep = true;
        }
        P.st[traj] = s;
    }
    append_active(P.idx[cur ^ 1], &P.count[cur ^ 1], traj, keep);  // whole warps take part in the ballot
}

// Rows still active when the host gives up (wall-clock watchdog).
template <int M>
__global__ void __launch_bounds__(kBlock) pl_abort(PropArgs A, PipeBufs P, int cur) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= P.count[cur]) return;
    const int32_t traj = P.idx[cur][slot];
    TrajState s = P.st[traj];
    traj_fail(A, s, traj, kWatchdog);
    P.st[traj] = s;
}

// ------------------------------------------------------------------- host
size_t pipeline_bytes(int64_t cap) {
    PipeBufs P{};
    pipeline_carve(P, nullptr, cap);
    return (size_t)(uintptr_t)P.dcount + 2 * sizeof(int32_t) + 256;
}

void pipeline_carve(PipeBufs& P, void* base, int64_t cap) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        off = (off + 255) & ~(size_t)255;
        char* p = (char*)base + off;
        off += bytes;
        return (void*)p;
    };
    const size_t c = (size_t)cap;
    P.cap = cap;
    P.st = (TrajState*)take(c * sizeof(TrajState));
    P.idx[0] = (int32_t*)take(c * 4);
    P.idx[1] = (int32_t*)take(c * 4);
    P.count = (int32_t*)take(2 * 4);
    P.k = (double*)take((size_t)kStageBufs * 6 * c * 8);
    P.sp = (double*)take(6 * c * 8);
    P.sc = (double*)take(2 * c * 8);
    P.fr = (double*)take(12 * c * 8);
    P.sun = (double*)take(3 * c * 8);
    P.part = (double*)take(3 * c * 8);
    P.agrav = (double*)take(3 * c * 8);
    P.adrag = (double*)take(3 * c * 8);
    P.jd = (double*)take(c * 8);
    P.amcd = (double*)take(2 * c * 8);
    P.skip = (int32_t*)take(c * 4);
    P.bad = (int32_t*)take(c * 4);
    P.dlist[0] = (int32_t*)take(c * 4);
    P.dlist[1] = (int32_t*)take(c * 4);
    P.ef = (double*)take(3 * c * 8);
    P.agx = (double*)take(3 * c * 8);
    P.fall = (int32_t*)take(c * 4);
    P.flist = (int32_t*)take(c * 4);
    P.fcount = (int32_t*)take(4);
    P.dcount = (int32_t*)take(2 * 4);  // last: pipeline_bytes measures up to it
}

template <int M>
static cudaError_t run(const PropArgs& A, const PipeBufs& P, cudaStream_t user, double max_seconds,
                       int gthreads, int gslots, KernelTimes* times) {
    using T = Tab<M>;
    // the dense stage: the end-of-step derivative of sampled segments and of
    // the eclipse coordinator's Hermite scan
    const bool dense = (A.out_mode != kOutFinalEci || A.force.srp) && !T::FSAL;
    const int stages = T::S + (dense ? 1 : 0);
    const int blocks = (int)((A.n + kBlock - 1) / kBlock);
    constexpr int kLanesHigh = BQP_DRAG_LANES_HIGH, kLanesLow = BQP_DRAG_LANES_LOW;
    const int dblocks_hi = (int)((A.n * kLanesHigh + kBlock - 1) / kBlock);
    const int dblocks_lo = (int)((A.n * kLanesLow + kBlock - 1) / kBlock);
    const int nt = gslots == 1 || gslots == 2 ? gslots : 4;
    auto gker = nt == 1 ? pl_gravity<1> : (nt == 2 ? pl_gravity<2> : pl_gravity<4>);
    if (gthreads > 256) gthreads = 256;
    if (gthreads < 32) gthreads = 32;
    gthreads = gthreads / 32 * 32;
    // column groups need room for their partial sums next to the table
    int gparts = kGravityPartsMax;
    // with the surrogate, the exact stage covers only the degrees it leaves out
    const bool sur = A.sur.P != nullptr;
    const GravTable GT = sur ? A.sur.low : A.grav;
    size_t smem = gravity_smem_bytes(GT, gthreads, nt, gparts);
    if (smem > kSmemPerBlock) {
        gparts = 1;
        smem = gravity_smem_bytes(GT, gthreads, nt, gparts);
    }
    // the surrogate's residual check also runs the whole exact field
    const bool check = sur && A.sur.check > 0.0;
    int gparts_full = kGravityPartsMax;
    size_t smem_full = 0;
    if (check) {
        smem_full = gravity_smem_bytes(A.sur.full, gthreads, nt, gparts_full);
        if (smem_full > kSmemPerBlock) {
            gparts_full = 1;
            smem_full = gravity_smem_bytes(A.sur.full, gthreads, nt, gparts_full);
        }
    }
    cudaError_t e = cudaFuncSetAttribute(gker, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(smem > smem_full ? smem : smem_full));
    if (e != cudaSuccess) return e;
    if (A.force.fit) {
        // the fixed-node fits: the same table for every context, ordered on
        // the caller's stream before this call's kernels
        if (!A.fit_host) return cudaErrorInvalidValue;
        e = cudaMemcpyToSymbolAsync(jb::c_fixed_fit, A.fit_host, sizeof(jb::JbFit), 0, cudaMemcpyHostToDevice, user);
        if (e != cudaSuccess) return e;
    }
    // one CTA per SM (the table fills shared memory); each takes an equal
    // share of the active slots, NT per thread
    int gblocks = device_sm_count();
    if (gblocks > A.n) gblocks = (int)A.n;
    if (gblocks < 1) gblocks = 1;

    // private stream ordered after the caller's stream (graphs need a
    // capturable stream)
    cudaStream_t st;
    e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
    cudaEvent_t ev_in, ev_out, ev_cnt;
    cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev_cnt, cudaEventDisableTiming);
    cudaEventRecord(ev_in, user);
    cudaStreamWaitEvent(st, ev_in, 0);
    int32_t* h_count = nullptr;
    cudaMallocHost(&h_count, sizeof(int32_t));

    cudaMemsetAsync(P.count, 0, 2 * sizeof(int32_t), st);
    if (check) cudaMemsetAsync(P.fall, 0, (size_t)A.n * sizeof(int32_t), st);
    pl_init<M><<<blocks, kBlock, 0, st>>>(A, P);

    // instrumentation: an event-record node on each side of every timed
    // kernel of the graph; the host sums the durations after each replay
    std::vector<cudaEvent_t> evs;
    std::vector<int> ev_class;  // class of the kernel between evs[2i] and evs[2i+1]
    auto timed = [&](int cls, auto&& launch) {
        if (!times) {
            launch();
            return;
        }
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecordWithFlags(a, st, cudaEventRecordExternal);
        launch();
        cudaEventRecordWithFlags(b, st, cudaEventRecordExternal);
        evs.push_back(a);
        evs.push_back(b);
        ev_class.push_back(cls);
    };
    // one graph = two attempts (active list 0 -> 1 -> 0)
    auto enqueue_attempt = [&](int cur, int timed_out) {
        for (int s = 0; s < stages; ++s) {
            if (A.force.drag) cudaMemsetAsync(P.dcount, 0, 2 * sizeof(int32_t), st);
            timed(kKcPrep, [&] { pl_prep<M><<<blocks, kBlock, 0, st>>>(A, P, cur, s); });
            if (A.force.gravity_on)
                timed(kKcGravity, [&] {
                    gker<<<gblocks, gthreads, smem, st>>>(GT, gparts, P, cur, P.agrav, nullptr, nullptr);
                    if (sur) {
                        pl_earth_fixed<<<blocks, kBlock, 0, st>>>(P, cur);
                        launch_surrogate_stage(A.sur, &P.count[cur], A.n, P.ef, P.agrav, 1, P.cap, st);
                        if (check && s == 0) {
                            // the exact field of every evaluated row, then the verdicts
                            cudaMemsetAsync(P.fcount, 0, sizeof(int32_t), st);
                            gker<<<gblocks, gthreads, smem_full, st>>>(A.sur.full, gparts_full, P, cur, P.agx,
                                                                      nullptr, nullptr);
                            pl_sur_check<<<blocks, kBlock, 0, st>>>(P, cur, A.sur.check);
                        } else if (check) {
                            // the rows on the exact field for this step
                            gker<<<gblocks, gthreads, smem_full, st>>>(A.sur.full, gparts_full, P, cur, P.agrav,
                                                                      P.flist, P.fcount);
                        }
                    }
                });
            if (A.force.drag)
                timed(kKcDrag, [&] {
                    if (A.force.atm_model == 4)
                        pl_drag<kLanesHigh, kLanesLow><<<dblocks_hi + dblocks_lo, kBlock, 0, st>>>(A.force, P,
                                                                                                 dblocks_hi);
                    else
                        pl_drag_coarse<<<2 * blocks, kBlock, 0, st>>>(A.force, P, blocks);
                });
        }
        timed(kKcControl, [&] { pl_control<M><<<blocks, kBlock, 0, st>>>(A, P, cur, dense ? 1 : 0, timed_out); });
    };
    auto collect = [&]() {
        for (size_t i = 0; i < ev_class.size(); ++i) {
            float ms = 0.0f;
            if (cudaEventElapsedTime(&ms, evs[2 * i], evs[2 * i + 1]) == cudaSuccess) {
                times->ms[ev_class[i]] += ms;
                times->launches[ev_class[i]] += 1;
            }
        }
    };
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        enqueue_attempt(0, 0);
        enqueue_attempt(1, 0);
        e = cudaStreamEndCapture(st, &graph);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
    const auto t_start = std::chrono::steady_clock::now();
    // host loop: replay, keep one replay in flight ahead of the count check
    int64_t replays = 0;
    bool done = false;
    while (e == cudaSuccess && !done) {
        e = cudaGraphLaunch(exec, st);
        if (e != cudaSuccess) break;
        cudaMemcpyAsync(h_count, &P.count[0], sizeof(int32_t), cudaMemcpyDeviceToHost, st);
        cudaEventRecord(ev_cnt, st);
        if (times) {
            // no replay in flight while the events of this one are read
            e = cudaEventSynchronize(ev_cnt);
            if (e != cudaSuccess) break;
            collect();
        }
        e = cudaGraphLaunch(exec, st);  // speculative: cheap when nothing is active
        if (e != cudaSuccess) break;
        e = cudaEventSynchronize(ev_cnt);
        if (times && e == cudaSuccess) {
            e = cudaStreamSynchronize(st);
            if (e == cudaSuccess) collect();
        }
        replays += 2;
        if (*h_count == 0) done = true;
        const double elapsed =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
        if (!done && max_seconds > 0.0 && elapsed > max_seconds) {
            cudaStreamSynchronize(st);
            pl_abort<M><<<blocks, kBlock, 0, st>>>(A, P, 0);
            done = true;
        }
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaEventRecord(ev_out, st);
    cudaStreamWaitEvent(user, ev_out, 0);
    cudaStreamSynchronize(st);
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaFreeHost(h_count);
    for (cudaEvent_t ev : evs) cudaEventDestroy(ev);
    cudaEventDestroy(ev_in);
    cudaEventDestroy(ev_out);
    cudaEventDestroy(ev_cnt);
    cudaStreamDestroy(st);
    return e;
}

cudaError_t launch_pipeline(const PropArgs& A, const PipeBufs& P, int method, cudaStream_t st, double max_seconds,
                            int gravity_threads, int gravity_slots, KernelTimes* times) {
    if (A.n <= 0) return cudaSuccess;
    if (gravity_threads <= 0) gravity_threads = 256;
    switch (method) {
        case kDopri5: return run<kDopri5>(A, P, st, max_seconds, gravity_threads, gravity_slots, times);
        case kDop853: return run<kDop853>(A, P, st, max_seconds, gravity_threads, gravity_slots, times);
        case kDopri5Compat:
            return run<kDopri5Compat>(A, P, st, max_seconds, gravity_threads, gravity_slots, times);
        case kVern7: return run<kVern7>(A, P, st, max_seconds, gravity_threads, gravity_slots, times);
        case kVern9: return run<kVern9>(A, P, st, max_seconds, gravity_threads, gravity_slots, times);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace bqp
