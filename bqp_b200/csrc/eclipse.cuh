// Binary-eclipse solar radiation pressure: the geometry and bounds of the
// reference's eclipse coordinator (lightyear_odeint_rs/src/eclipse.rs,
// eclipse_coordinator.rs), per trajectory on the device.
//
// A row with SRP integrates in legs that hold the eclipse side fixed.  After
// every accepted step the step's cubic Hermite path (positions and
// velocities from the step's ends) is scanned for a crossing of the Earth's
// shadow cylinder; traj.cuh sequences the legs that replay and commit one.
// This file holds the per-step pieces: the scan and its bounds.
#pragma once
#include <cstdint>
#include <cstring>

#include "kernels.cuh"

namespace bqp {

constexpr double kEclMaxSepKm = 1.0e-6;         // eclipse.rs:39 bracket resolution (1 mm)
constexpr double kEclSpeedCap = 20.0;           // eclipse.rs:50 km/s
constexpr double kEclRadiusMin = 6000.0;        // eclipse.rs:45 km
constexpr double kEclRadiusCap = 50000.0;       // eclipse.rs:46 km
constexpr double kEclRootUncKm = 1.0e-4;        // eclipse_coordinator.rs:93
constexpr double kEclOldSideMarginKm = 2.5e-5;  // eclipse_coordinator.rs:94
constexpr int kEclProofRestarts = 2;            // eclipse_coordinator.rs:110
constexpr double kEclPostRootSafety = 16.0;     // eclipse_coordinator.rs:117
constexpr double kEclMinDecisiveKm = 1.0e-9;    // eclipse_coordinator.rs:130
constexpr double kEclRefineStepS = 10.0;        // eclipse_coordinator.rs:254
constexpr int64_t kEclMaxSplits = 4096;         // eclipse_coordinator.rs:256
constexpr double kEclHcarryMinDtMax = 60.0;     // integrator.rs HCARRY_UNCLAMPED_DT_MAX_S
constexpr int64_t kEclMaxIter = 500000;         // integrator.rs:185
// Upper bound of the analytic Sun series' direction rate, rad/day: the
// ecliptic longitude advances at most 0.98565 + 1.955 x 0.0172 deg/day
// (mean motion and the equation of centre) = 0.01779 rad/day.  A catalogue
// takes the supremum over its own linear pieces (ForceParams::sun_rate).
constexpr double kSunRateAnalytic = 0.0185;
constexpr int kEclScanDepth = 64;               // bisection levels of one scan (binary64 runs out first)

// Legs of the coordinator.
enum EclLeg : int32_t { kLegMain = 0, kLegRefine = 1, kLegProof = 2, kLegWindow = 3 };

// Coordinator state of one SRP row (global memory, one per trajectory).
struct EclState {
    double root_t, root_err;     // last committed root and its rebase transport error
    double a, b;                 // crossing step of the main leg (the refine leg's span)
    double b2;                   // end of the refined crossing step
    double br_told, br_tnew;     // refined bracket of the crossing
    double anchor, proof_old_t;  // old-side proof anchor and end
    double fch;                  // the leg's final controller step (step-size carry)
    int32_t have_root, leg, br_old, br_new, restarts, idx_base;
    int64_t splits, iters;
};

__host__ __device__ __forceinline__ double ulps_up(double v, uint64_t k) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double(__double_as_longlong(v) + (long long)k);
#else
    uint64_t b;
    memcpy(&b, &v, 8);
    b += k;
    memcpy(&v, &b, 8);
    return v;
#endif
}

// One representable value outward (eclipse_coordinator.rs:570-588).
__device__ __forceinline__ bool ecl_outward(double v, double* out) {
    if (!(isfinite(v) && v >= 0.0)) return false;
    if (v == 0.0) {
        *out = 0.0;
        return true;
    }
    const double r = ulps_up(v, 1);
    if (!isfinite(r)) return false;
    *out = r;
    return true;
}

__device__ __forceinline__ double dist3(const double* a, const double* b) {
    const double dx = b[0] - a[0], dy = b[1] - a[1], dz = b[2] - a[2];
    return sqrt(fma(dx, dx, fma(dy, dy, dz * dz)));
}

// Position, velocity and Sun of a row at solver time t; the arc's geometry.
struct EclGeo {
    const ForceParams* fp;
    double jd0;

    __device__ bool sun(double t, double* o) const {
        if (!isfinite(t)) return false;
        const double jd = utc_jd_at(jd0, t);
        if (fp->eph_sun.n > 0 && !(jd >= fp->eph_sun.jd_start && jd <= fp->eph_sun.jd_end)) return false;
        sun_at(fp->eph_sun, jd, o);
        const double n2 = o[0] * o[0] + o[1] * o[1] + o[2] * o[2];
        return isfinite(n2) && n2 > 0.0;
    }
    // rhs.rs:4788-4866: direction rate x elapsed days, one value outward
    __device__ int32_t sun_angle(double a, double b, double* out) const {
        if (!isfinite(a) || !isfinite(b)) return kEclGeometry;
        if (fp->eph_sun.n > 0) {
            const double ja = utc_jd_at(jd0, a), jb = utc_jd_at(jd0, b);
            const double lo = fp->eph_sun.jd_start, hi = fp->eph_sun.jd_end;
            if (!(ja >= lo && ja <= hi && jb >= lo && jb <= hi)) return kEclGeometry;
        }
        const double rate = fp->sun_rate;
        if (!(isfinite(rate) && rate >= 0.0)) return kEclGeometry;
        const double bound = rate * (fabs(b - a) / 86400.0);
        if (!isfinite(bound)) return kEclGeometry;
        if (bound == 0.0) {
            *out = 0.0;
            return kOk;
        }
        const double r = ulps_up(bound, 1);
        if (!isfinite(r)) return kEclGeometry;
        *out = r;
        return kOk;
    }
    // eclipse_coordinator.rs:590-596: speed cap x dt + diameter cap x Sun sweep
    __device__ int32_t replay_unc(double t0, double t1, double* out) const {
        double dtb, dia, ang, axis;
        if (!ecl_outward(kEclSpeedCap * fabs(t1 - t0), &dtb)) return kEclGeometry;
        if (!ecl_outward(2.0 * kEclRadiusCap, &dia)) return kEclGeometry;
        if (int32_t e = sun_angle(t0, t1, &ang)) return e;
        if (!ecl_outward(dia * ang, &axis)) return kEclGeometry;
        if (!ecl_outward(dtb + axis, out)) return kEclGeometry;
        return kOk;
    }
    // eclipse_coordinator.rs:598-631: farthest instant from old_t toward lim
    // whose replay uncertainty stays within maxb
    __device__ int32_t deepest(double old_t, double lim, double maxb, double* out) const {
        if (old_t == lim || !isfinite(lim) || !(isfinite(maxb) && maxb > 0.0)) return kEclNonProgress;
        double u;
        if (int32_t e = replay_unc(old_t, lim, &u)) return e;
        if (u <= maxb) {
            *out = lim;
            return kOk;
        }
        double inside = old_t, outside = lim;
        for (int i = 0; i < 64; ++i) {
            const double mid = inside + 0.5 * (outside - inside);
            if (mid == inside || mid == outside) break;
            if (int32_t e = replay_unc(old_t, mid, &u)) return e;
            if (u <= maxb) inside = mid;
            else outside = mid;
        }
        if (inside == old_t || !isfinite(inside)) return kEclNonProgress;
        *out = inside;
        return kOk;
    }
};

// eclipse_coordinator.rs:182-194
__device__ __forceinline__ int32_t ecl_decisive_margin(double err, double* out) {
    if (!(isfinite(err) && err >= 0.0)) return kEclGeometry;
    double sc;
    if (!ecl_outward(kEclPostRootSafety * err, &sc)) return kEclGeometry;
    *out = fmin(fmax(sc, kEclMinDecisiveKm), kEclMaxSepKm);
    return kOk;
}

// eclipse.rs:124-152 on a baseline state b plus delta d.
__device__ __forceinline__ bool ecl_envelope_of(const double* b, const double* d) {
    const double p0 = b[0] + d[0], p1 = b[1] + d[1], p2 = b[2] + d[2];
    const double v0 = b[3] + d[3], v1 = b[4] + d[4], v2 = b[5] + d[5];
    if (!(isfinite(p0) && isfinite(p1) && isfinite(p2) && isfinite(v0) && isfinite(v1) && isfinite(v2)))
        return false;
    const double r = sqrt(fma(p0, p0, fma(p1, p1, p2 * p2)));
    const double s = sqrt(fma(v0, v0, fma(v1, v1, v2 * v2)));
    return isfinite(r) && isfinite(s) && r >= kEclRadiusMin && r <= kEclRadiusCap && s <= kEclSpeedCap;
}

// ... on baseline + delta at solver time t.
__device__ __forceinline__ bool ecl_envelope(const Baseline& base, double bt0, const double* d, double t) {
    double b[6];
    baseline_state(base, t - bt0, b);
    const double p0 = b[0] + d[0], p1 = b[1] + d[1], p2 = b[2] + d[2];
    const double v0 = b[3] + d[3], v1 = b[4] + d[4], v2 = b[5] + d[5];
    if (!(isfinite(p0) && isfinite(p1) && isfinite(p2) && isfinite(v0) && isfinite(v1) && isfinite(v2)))
        return false;
    const double r = sqrt(fma(p0, p0, fma(p1, p1, p2 * p2)));
    const double s = sqrt(fma(v0, v0, fma(v1, v1, v2 * v2)));
    return isfinite(r) && isfinite(s) && r >= kEclRadiusMin && r <= kEclRadiusCap && s <= kEclSpeedCap;
}

// Side of baseline + delta at t (rhs.rs:4422-4444).
__device__ __forceinline__ int32_t ecl_side_at(const EclGeo& G, const Baseline& base, double bt0, const double* d,
                                               double t, int* side, double* margin) {
    double b[6], sun[3];
    baseline_state(base, t - bt0, b);
    const double p[3] = {b[0] + d[0], b[1] + d[1], b[2] + d[2]};
    if (!G.sun(t, sun)) return kEclGeometry;
    if (!shadow_cylinder(p, sun, G.fp->earth_radius, side, margin)) return kEclGeometry;
    return kOk;
}

// The accepted step's Hermite path (eclipse_coordinator.rs:313-361, 377-568).
struct EclPath {
    double p0[3], v0[3], p1[3], v1[3], t0, t1;

    __device__ int32_t at(double t, double* pos, double* vel) const {
        const double h = t1 - t0;
        if (!isfinite(h) || h == 0.0 || !isfinite(t)) return kEclNonProgress;
        const double tau = fmin(fmax((t - t0) / h, 0.0), 1.0);
        const double t2 = tau * tau, t3 = t2 * tau;
        const double h00 = 2.0 * t3 - 3.0 * t2 + 1.0, h10 = t3 - 2.0 * t2 + tau;
        const double h01 = -2.0 * t3 + 3.0 * t2, h11 = t3 - t2;
        const double g00 = (6.0 * t2 - 6.0 * tau) / h, g10 = 3.0 * t2 - 4.0 * tau + 1.0;
        const double g01 = (-6.0 * t2 + 6.0 * tau) / h, g11 = 3.0 * t2 - 2.0 * tau;
        for (int i = 0; i < 3; ++i) {
            pos[i] = h00 * p0[i] + h10 * h * v0[i] + h01 * p1[i] + h11 * h * v1[i];
            vel[i] = g00 * p0[i] + g10 * v0[i] + g01 * p1[i] + g11 * v1[i];
        }
        for (int i = 0; i < 3; ++i)
            if (!isfinite(pos[i]) || !isfinite(vel[i])) return kEclGeometry;
        return kOk;
    }
};

// One scan endpoint: time, position, velocity, side and boundary margin.
struct EclPoint {
    double t, p[3], v[3];
    int side;
    double margin;
};

__device__ __forceinline__ int32_t ecl_point(const EclGeo& G, const EclPath& H, double t, EclPoint* q) {
    if (!isfinite(t)) return kEclGeometry;
    q->t = t;
    if (int32_t e = H.at(t, q->p, q->v)) return e;
    double sun[3];
    if (!G.sun(t, sun)) return kEclGeometry;
    if (!shadow_cylinder(q->p, sun, G.fp->earth_radius, &q->side, &q->margin)) return kEclGeometry;
    return kOk;
}

// eclipse_coordinator.rs:499-547: control-polygon length of the Hermite
// path plus the swing of the Sun axis, eight values outward.
__device__ __forceinline__ int32_t ecl_motion_bound(const EclGeo& G, const EclPoint& a, const EclPoint& b,
                                                    double* out) {
    const double h = b.t - a.t;
    double c1[3], c2[3];
    for (int i = 0; i < 3; ++i) {
        c1[i] = a.p[i] + h * a.v[i] / 3.0;
        c2[i] = b.p[i] - h * b.v[i] / 3.0;
    }
    const double path = dist3(a.p, c1) + dist3(c1, c2) + dist3(c2, b.p);
    double m2 = 0.0;
    const double* pts[4] = {a.p, c1, c2, b.p};
    for (int k = 0; k < 4; ++k) {
        const double* p = pts[k];
        const double r2 = fma(p[0], p[0], fma(p[1], p[1], p[2] * p[2]));
        if (r2 > m2) m2 = r2;  // a NaN radius is discarded
    }
    const double maxr = sqrt(m2);
    double ang;
    if (int32_t e = G.sun_angle(a.t, b.t, &ang)) return e;
    const double bound = path + 2.0 * maxr * ang;
    if (!isfinite(bound)) return kEclGeometry;
    if (bound == 0.0) {
        *out = 0.0;
        return kOk;
    }
    const double r = ulps_up(bound, 8);
    if (!isfinite(r)) return kEclGeometry;
    *out = r;
    return kOk;
}

struct EclBracket {
    double t_old, t_new, bound;
    int old_side, new_side;
};

// First side change along the path in [t_a, t_b] (eclipse.rs:341-491):
// depth-first bisection at binary64 midpoints, earliest interval first,
// until the geometry motion across a bracket is at most kEclMaxSepKm; an
// interval whose end margins exceed its motion bound holds no crossing.
// The recursion runs on an explicit stack of right endpoints.
// `budget` caps the splits this call may take: a walk that needs more
// returns kEclDefer with nothing decided, for the warp-cooperative walk to
// redo from the start (the same result, sooner).
constexpr int32_t kEclDefer = -2;
static __device__ __noinline__ int32_t ecl_first_crossing(const EclGeo& G, const EclPath& H, double t_a, double t_b,
                                                   bool* found, EclBracket* br, int64_t budget = kEclMaxSplits,
                                                   const EclPoint* start = nullptr) {
    *found = false;
    if (t_a == t_b) return kEclNonProgress;
    double st_t[kEclScanDepth], st_b[kEclScanDepth];
    int sp = 0;
    int64_t splits_left = kEclMaxSplits;
    EclPoint L, R;
    if (start) L = *start;  // the point at t_a, already evaluated
    else if (int32_t e = ecl_point(G, H, t_a, &L)) return e;
    if (int32_t e = ecl_point(G, H, t_b, &R)) return e;
    bool inherited = false;
    double inh = 0.0;
    for (;;) {
        bool resolved = false;
        const double sep = dist3(L.p, R.p);
        if (!isfinite(sep)) return kEclGeometry;
        if (L.side == R.side && inherited && L.margin + R.margin > inh) {
            resolved = true;
        } else {
            double mb;
            if (int32_t e = ecl_motion_bound(G, L, R, &mb)) return e;
            if (!(isfinite(mb) && mb >= sep && mb >= 0.0)) return kEclBracket;
            if (L.side == R.side && L.margin + R.margin > mb) {
                resolved = true;
            } else if (mb <= kEclMaxSepKm && L.side != R.side) {
                br->t_old = L.t;
                br->t_new = R.t;
                br->old_side = L.side;
                br->new_side = R.side;
                br->bound = mb;
                *found = true;
                return kOk;
            } else {
                const double mid = L.t + 0.5 * (R.t - L.t);
                if (mid == L.t || mid == R.t || !isfinite(mid)) {
                    // adjacent binary64 instants: nothing representable between
                    if (L.side == R.side && mb <= 1.0e-6) resolved = true;
                    else return kEclNonProgress;
                } else {
                    if (splits_left == 0 || sp == kEclScanDepth) return kEclSplitLimit;
                    if (kEclMaxSplits - splits_left >= budget) return kEclDefer;
                    --splits_left;
                    st_t[sp] = R.t;
                    st_b[sp] = mb;
                    ++sp;
                    if (int32_t e = ecl_point(G, H, mid, &R)) return e;
                    inherited = true;
                    inh = mb;
                }
            }
        }
        if (resolved) {
            if (sp == 0) return kOk;
            --sp;
            L = R;
            if (int32_t e = ecl_point(G, H, st_t[sp], &R)) return e;
            inherited = true;
            inh = st_b[sp];
        }
    }
}

// CoordinatedEventHandler::on_step (eclipse_coordinator.rs:720-934), events
// off, before its scan: checks the accepted step [t0, t1] of a leg on side
// `fixed` (deltas y, derivatives d against baseline `base` from bt0), builds
// the step's Hermite path and the instant the scan starts from.
static __device__ __noinline__ int32_t ecl_step_pre(const EclGeo& G, const Baseline& base, double bt0, int fixed,
                                             const EclState& E, double t0, const double* y0, const double* d0,
                                             double t1, const double* y1, const double* d1, EclPath* H,
                                             double* from, EclPoint* start) {
    double b0[6], b1[6];
    baseline_state(base, t0 - bt0, b0);
    baseline_state(base, t1 - bt0, b1);
    if (!ecl_envelope_of(b0, y0) || !ecl_envelope_of(b1, y1)) return kEclEnvelope;
    for (int i = 0; i < 3; ++i) {
        H->p0[i] = b0[i] + y0[i];
        H->v0[i] = b0[3 + i] + d0[i];
        H->p1[i] = b1[i] + y1[i];
        H->v1[i] = b1[3 + i] + d1[i];
    }
    H->t0 = t0;
    H->t1 = t1;
    EclPoint q;
    if (int32_t e = ecl_point(G, *H, t0, &q)) return e;
    const bool certified = E.have_root && E.root_t == t0;
    if (q.side != fixed && !certified) return kEclChatter;
    *from = t0;
    if (certified) {
        // inside the committed root's uncertainty the side is not resolvable:
        // scan from the deepest instant the root bound covers, where it must
        // read the committed side decisively
        double edge, dm;
        if (int32_t e = G.deepest(t0, t1, kEclRootUncKm, &edge)) return e;
        if (int32_t e = ecl_point(G, *H, edge, &q)) return e;
        if (int32_t e = ecl_decisive_margin(E.root_err, &dm)) return e;
        if (q.side != fixed || q.margin <= dm) return kEclChatter;
        *from = edge;
    }
    *start = q;  // the scan's first end point
    return kOk;
}

// ------------------------------------------------ warp-cooperative scan
// The same depth-first bisection as ecl_first_crossing, with the points and
// motion bounds it may need evaluated 32 at a time.  Whenever the walk
// splits the root of its store, the warp fills the store with that node's
// whole 5-level subtree: the 31 midpoints (one lane each, every lane
// descending the binary64 midpoint chain the serial walk would form) and the
// bounds of the 62 sub-intervals (two per lane).  Every lane then walks the
// subtree with the serial rules on the shared copy, so decisions, split
// counts, the stack and the errors reported are the serial walk's; only a
// split at the subtree's bottom level, or a return to a node of an older
// store, costs another evaluation round.  A few rows near grazing geometry
// scan thousands of points per step; serially the whole batch waits for
// them.
constexpr int kEclGrid = 32;  // grid positions 0..32 of one store; nodes by heap index 1..63

struct EclWarpStore {
    double t[kEclGrid + 1], p[kEclGrid + 1][3], v[kEclGrid + 1][3], m[kEclGrid + 1];
    int32_t side[kEclGrid + 1], pst[kEclGrid + 1];  // point status; kEclBadMid: no representable midpoint
    double bnd[2 * kEclGrid];
    int32_t bst[2 * kEclGrid];
    int32_t fl[2 * kEclGrid];  // the walk's tests of each node, evaluated with the bounds (kNode*)
    double st_t[kEclScanDepth], st_inh[kEclScanDepth];  // pending right siblings: end time, parent bound
    int32_t st_h[kEclScanDepth], st_gen[kEclScanDepth];
};
constexpr int32_t kEclBadMid = -1;
// Node tests: end points on one side; chord not finite; certified by the
// parent's bound (how the walk first tries every node below a split);
// certified by its own bound; bound below the chord or not finite; a bracket
// (own bound within the resolution, sides differ); bound within 1 mm (the
// adjacent-instant rule).
enum : int32_t {
    kNodeSame = 1, kNodeSepBad = 2, kNodeCertInh = 4, kNodeCertOwn = 8, kNodeBadBound = 16, kNodeFound = 32,
    kNodeFine = 64
};

__device__ __forceinline__ void ecl_store_point(EclWarpStore& W, int pos, const EclPoint& q) {
    W.t[pos] = q.t;
    for (int i = 0; i < 3; ++i) {
        W.p[pos][i] = q.p[i];
        W.v[pos][i] = q.v[i];
    }
    W.m[pos] = q.margin;
    W.side[pos] = q.side;
    W.pst[pos] = kOk;
}

__device__ __forceinline__ EclPoint ecl_load_point(const EclWarpStore& W, int pos) {
    EclPoint q;
    q.t = W.t[pos];
    for (int i = 0; i < 3; ++i) {
        q.p[i] = W.p[pos][i];
        q.v[i] = W.v[pos][i];
    }
    q.margin = W.m[pos];
    q.side = W.side[pos];
    return q;
}

// Grid positions [a, b] of node h (heap index, level d = floor(log2 h)).
__device__ __forceinline__ void ecl_node_span(int h, int* a, int* b) {
    const int d = 31 - __clz(h);
    const int w = kEclGrid >> d;
    *a = (h - (1 << d)) * w;
    *b = *a + w;
}

// Fill positions 1..31, and the bounds and tests of nodes 2..63, below the
// store's root (positions 0 and 32 hold its ends; root_mb is its bound).
// All lanes.
static __device__ __noinline__ void ecl_expand(const EclGeo& G, const EclPath& H, EclWarpStore& W, int lane,
                                               double root_mb) {
    if (lane >= 1) {
        // the midpoint chain from the root down to this lane's position
        double lo = W.t[0], hi = W.t[kEclGrid];
        int plo = 0, phi = kEclGrid;
        for (;;) {
            const int pm = (plo + phi) >> 1;
            const double mid = lo + 0.5 * (hi - lo);
            if (mid == lo || mid == hi || !isfinite(mid)) {
                W.pst[lane] = kEclBadMid;
                break;
            }
            if (pm == lane) {
                EclPoint q;
                const int32_t e = ecl_point(G, H, mid, &q);
                ecl_store_point(W, lane, q);
                W.t[lane] = mid;
                W.pst[lane] = e;
                break;
            }
            if (lane < pm) {
                hi = mid;
                phi = pm;
            } else {
                lo = mid;
                plo = pm;
            }
        }
    }
    __syncwarp();
    for (int h = 2 + lane; h < 2 * kEclGrid; h += 32) {
        int a, b;
        ecl_node_span(h, &a, &b);
        if (W.pst[a] == kOk && W.pst[b] == kOk) {
            const EclPoint qa = ecl_load_point(W, a), qb = ecl_load_point(W, b);
            W.bst[h] = ecl_motion_bound(G, qa, qb, &W.bnd[h]);
        } else {
            W.bst[h] = kEclBadMid;  // under a point the walk never passes
        }
    }
    __syncwarp();
    // the walk's tests of every node, each under its parent's bound
    for (int h = 2 + lane; h < 2 * kEclGrid; h += 32) {
        int a, b;
        ecl_node_span(h, &a, &b);
        int32_t f = 0;
        if (W.pst[a] == kOk && W.pst[b] == kOk) {
            const double sep = dist3(W.p[a], W.p[b]);
            const double msum = W.m[a] + W.m[b];
            const double inh = h < 4 ? root_mb : W.bnd[h >> 1];
            const bool same = W.side[a] == W.side[b];
            if (same) f |= kNodeSame;
            if (!isfinite(sep)) f |= kNodeSepBad;
            if (same && msum > inh) f |= kNodeCertInh;
            if (W.bst[h] == kOk) {
                const double mb = W.bnd[h];
                if (!(isfinite(mb) && mb >= sep && mb >= 0.0)) f |= kNodeBadBound;
                if (same && msum > mb) f |= kNodeCertOwn;
                if (mb <= kEclMaxSepKm && !same) f |= kNodeFound;
                if (mb <= 1.0e-6) f |= kNodeFine;
            }
        }
        W.fl[h] = f;
    }
    __syncwarp();
}

// One node's verdict under the serial rules.
enum : int32_t { kVerdictResolved = 0, kVerdictFound = 1, kVerdictSplit = 2 };
struct EclNodeTest {
    int32_t err, verdict;
    double mb;
};

// ... from its end points, the bound computed when needed (a store's root)
__device__ __forceinline__ EclNodeTest ecl_node_test_points(const EclGeo& G, const EclPoint& L, const EclPoint& R,
                                                            bool inherited, double inh) {
    const double sep = dist3(L.p, R.p);
    if (!isfinite(sep)) return {kEclGeometry, 0, 0.0};
    const bool same = L.side == R.side;
    if (same && inherited && L.margin + R.margin > inh) return {kOk, kVerdictResolved, 0.0};
    double mb;
    if (int32_t e = ecl_motion_bound(G, L, R, &mb)) return {e, 0, 0.0};
    if (!(isfinite(mb) && mb >= sep && mb >= 0.0)) return {kEclBracket, 0, 0.0};
    if (same && L.margin + R.margin > mb) return {kOk, kVerdictResolved, mb};
    if (mb <= kEclMaxSepKm && !same) return {kOk, kVerdictFound, mb};
    const double mid = L.t + 0.5 * (R.t - L.t);
    if (mid == L.t || mid == R.t || !isfinite(mid)) {
        if (same && mb <= 1.0e-6) return {kOk, kVerdictResolved, mb};
        return {kEclNonProgress, 0, 0.0};
    }
    return {kOk, kVerdictSplit, mb};
}

// ... from the store's precomputed tests (a node below the root, reached
// through its parent's split)
__device__ __forceinline__ EclNodeTest ecl_node_test_store(const EclWarpStore& W, int h, int a, int b) {
    const int32_t f = W.fl[h];
    if (f & kNodeSepBad) return {kEclGeometry, 0, 0.0};
    if (f & kNodeCertInh) return {kOk, kVerdictResolved, 0.0};
    if (W.bst[h] != kOk) return {W.bst[h], 0, 0.0};
    const double mb = W.bnd[h];
    if (f & kNodeBadBound) return {kEclBracket, 0, 0.0};
    if (f & kNodeCertOwn) return {kOk, kVerdictResolved, mb};
    if (f & kNodeFound) return {kOk, kVerdictFound, mb};
    bool no_mid;
    if (b - a > 1) {
        no_mid = W.pst[(a + b) >> 1] == kEclBadMid;
    } else {
        const double mid = W.t[a] + 0.5 * (W.t[b] - W.t[a]);
        no_mid = mid == W.t[a] || mid == W.t[b] || !isfinite(mid);
    }
    if (no_mid) {
        if ((f & kNodeSame) && (f & kNodeFine)) return {kOk, kVerdictResolved, mb};
        return {kEclNonProgress, 0, 0.0};
    }
    return {kOk, kVerdictSplit, mb};
}

// Earliest crossing of the path in [t_a, t_b]: every lane of the warp calls
// it with the same arguments and returns the same result.
static __device__ __noinline__ int32_t ecl_first_crossing_warp(const EclGeo& G, const EclPath& H, double t_a,
                                                               double t_b, EclWarpStore& W, bool* found,
                                                               EclBracket* br, const EclPoint* start = nullptr) {
    const int lane = threadIdx.x & 31;
    *found = false;
    if (t_a == t_b) return kEclNonProgress;
    {
        EclPoint q;
        int32_t e = kOk;
        if (lane == 0) {
            if (start) q = *start;
            else e = ecl_point(G, H, t_a, &q);
        } else if (lane == 1) {
            e = ecl_point(G, H, t_b, &q);
        }
        if (lane < 2) {
            ecl_store_point(W, lane == 0 ? 0 : kEclGrid, q);
            W.pst[lane == 0 ? 0 : kEclGrid] = e;
        }
        __syncwarp();
        if (W.pst[0] != kOk) return W.pst[0];
        if (W.pst[kEclGrid] != kOk) return W.pst[kEclGrid];
    }
    int gen = 0, sp = 0, h = 1;
    bool inherited = false;
    double inh = 0.0;
    int64_t splits_left = kEclMaxSplits;
    for (;;) {
        int a, b;
        ecl_node_span(h, &a, &b);
        const EclNodeTest T = h == 1
                                  ? ecl_node_test_points(G, ecl_load_point(W, a), ecl_load_point(W, b), inherited, inh)
                                  : ecl_node_test_store(W, h, a, b);
        if (T.err) return T.err;
        if (T.verdict == kVerdictFound) {
            br->t_old = W.t[a];
            br->t_new = W.t[b];
            br->old_side = W.side[a];
            br->new_side = W.side[b];
            br->bound = T.mb;
            *found = true;
            return kOk;
        }
        if (T.verdict == kVerdictSplit) {
            if (splits_left == 0 || sp == kEclScanDepth) return kEclSplitLimit;
            --splits_left;
            const double r_t = W.t[b];
            if (h == 1 || b - a == 1) {
                if (b - a == 1) {
                    // a bottom-level node becomes the root of a new store
                    const EclPoint L = ecl_load_point(W, a), R = ecl_load_point(W, b);
                    __syncwarp();
                    if (lane == 0) {
                        ecl_store_point(W, 0, L);
                        ecl_store_point(W, kEclGrid, R);
                    }
                    __syncwarp();
                    ++gen;
                    h = 1;
                    a = 0;
                    b = kEclGrid;
                }
                ecl_expand(G, H, W, lane, T.mb);
            }
            if (lane == 0) {
                W.st_t[sp] = r_t;
                W.st_inh[sp] = T.mb;
                W.st_h[sp] = 2 * h + 1;
                W.st_gen[sp] = gen;
            }
            __syncwarp();
            ++sp;
            const int pm = (a + b) >> 1;
            if (W.pst[pm] != kOk) return W.pst[pm];
            h = 2 * h;
            inherited = true;
            inh = T.mb;
            continue;
        }
        // resolved: the next pending right sibling
        if (sp == 0) return kOk;
        --sp;
        const int ph = W.st_h[sp], pg = W.st_gen[sp];
        const double pt = W.st_t[sp], pinh = W.st_inh[sp];
        if (pg == gen) {
            h = ph;
        } else {
            // a sibling from an older store: a new store rooted at it, from
            // this node's right end to the sibling's (evaluated again: the
            // same bits)
            const EclPoint R = ecl_load_point(W, b);
            EclPoint q;
            const int32_t e = ecl_point(G, H, pt, &q);
            __syncwarp();
            if (lane == 0) {
                ecl_store_point(W, 0, R);
                ecl_store_point(W, kEclGrid, q);
                W.pst[kEclGrid] = e;
            }
            __syncwarp();
            if (e != kOk) return e;
            ++gen;
            h = 1;
        }
        inherited = true;
        inh = pinh;
    }
}

}  // namespace bqp
