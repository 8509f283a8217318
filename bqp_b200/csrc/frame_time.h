// IAU 2006/2000A Earth-fixed frame: the per-stage GCRS->ITRS rotation from
// 1800 s segments (satpy_core frame_time/authority.rs), shared by the host
// segment builder (frame_time.cpp), the kernels and the C ABI.
//
// Time is continuous TAI seconds from 0h TAI of MJD 41684 (1973-01-02),
// the origin of the reference's sealed frame authority (authority.rs:92,
// 1162-1190).  A segment is keyed by (j, k): j the leap interval holding the
// instant, k the whole 1800 s widths from that interval's start, the
// interval's trailing remainder absorbed by its last segment
// (authority.rs:416-470).  Inside a segment
//   R(dt) = cos(theta)(M0 + dt K0) + sin(theta)(M1 + dt K1) + (M2 + dt K2),
//   theta(dt) = b0 + dt (b1 + dt (b2 + dt b3)),
// dt from the segment centre, and the ITRS angular velocity comes from the
// exact derivative of that interpolant (authority.rs:682-794).
#pragma once
#include <cmath>
#include <cstdint>

#ifndef BQP_HD
#ifdef __CUDACC__
#define BQP_HD __host__ __device__ __forceinline__
#else
#define BQP_HD inline
#endif
#endif

namespace bqp {
namespace ft {

constexpr double kSegWidth = 1800.0;
constexpr int32_t kOriginMjd = 41684;     // 1973-01-02
constexpr double kDaySec = 86400.0;
constexpr double kDjm0 = 2400000.5;
constexpr int kMaxIntervals = 48;         // leap intervals the table can hold

// Products and sums written out so that nvcc does not contract them into
// FMAs: the host restatement and the kernels then round alike.
#ifdef __CUDA_ARCH__
BQP_HD double mul_rn(double a, double b) { return __dmul_rn(a, b); }
BQP_HD double add_rn(double a, double b) { return __dadd_rn(a, b); }
#else
BQP_HD double mul_rn(double a, double b) { return a * b; }
BQP_HD double add_rn(double a, double b) { return a + b; }
#endif

// One canonical segment (authority.rs:224-236).
struct FrameSeg {
    double m[3][9];    // row-major 3x3 each: M0, M1, M2
    double k[3][9];    // their centred slopes, per second
    double b[4];       // theta cubic in dt seconds
    double centre;     // continuous TAI seconds
    double delta_at;   // TAI - UTC over the segment
};

// A per-stage rotation: r maps GCRS to ITRS, w is ITRS's angular velocity
// relative to GCRS, in GCRS (rad/s).
struct FrameRot {
    double r[9];
    double w[3];
};

// Leap intervals of the span: start (continuous TAI seconds) and TAI - UTC
// from that instant on (authority.rs:192-220).
struct FrameIntervals {
    int32_t n;
    double start[kMaxIntervals];
    double delta_at[kMaxIntervals];
    double span_end;   // exclusive end of the span, continuous TAI seconds
};

// The device view the kernels read: segments sorted by key.
struct FrameTab {
    int32_t mode;               // 0: GMST z-rotation; 1: these segments
    int32_t nseg;
    const FrameSeg* seg;
    const int64_t* key;
    const FrameIntervals* ivl;
};

BQP_HD int64_t seg_key(int32_t j, int64_t k) { return ((int64_t)j << 40) | k; }

// (j, k) of an instant; false outside the span (authority.rs:416-470).
BQP_HD bool segment_index(const FrameIntervals& I, double tai, int32_t* j_out, int64_t* k_out) {
    if (!(tai == tai) || tai >= I.span_end || I.n <= 0) return false;
    if (!(tai - tai == 0.0)) return false;  // infinite
    int32_t j = -1;
    for (int32_t q = I.n - 1; q >= 0; --q)
        if (I.start[q] <= tai) { j = q; break; }
    if (j < 0) return false;
    const double start = I.start[j];
    double kf = floor((tai - start) / kSegWidth);
    int64_t k = kf < 0.0 ? 0 : (int64_t)kf;
    if (j + 1 < I.n) {
        const int64_t whole = (int64_t)floor((I.start[j + 1] - start) / kSegWidth);
        if (whole > 0 && k >= whole) k = whole - 1;
    }
    *j_out = j;
    *k_out = k;
    return true;
}

// Slot of the segment holding `tai` in a sorted key table, or -1.
BQP_HD int32_t segment_slot(const FrameTab& T, double tai) {
    int32_t j;
    int64_t k;
    if (!T.ivl || !segment_index(*T.ivl, tai, &j, &k)) return -1;
    const int64_t key = seg_key(j, k);
    if (T.nseg <= 0) return -1;
    // a table built for one span holds consecutive keys: the key's offset
    // from the first one is its slot (one load); otherwise binary search
    const int64_t g = key - T.key[0];
    if (g >= 0 && g < T.nseg && T.key[g] == key) return (int32_t)g;
    int32_t lo = 0, hi = T.nseg - 1;
    while (lo <= hi) {
        const int32_t mid = (lo + hi) >> 1;
        const int64_t v = T.key[mid];
        if (v == key) return mid;
        if (v < key) lo = mid + 1;
        else hi = mid - 1;
    }
    return -1;
}

// The rotation and ITRS angular velocity at `tai` inside segment `S`
// (authority.rs:682-794): one sin/cos, the 3x3 blend with its exact
// derivative, and w from the skew part of Rdot R^T (passive convention
// Rdot R^T = -[w_itrs x]), rotated back to GCRS.
BQP_HD void rotation_at(const FrameSeg& S, double tai, FrameRot& out) {
    const double dt = tai - S.centre;
    const double theta = S.b[0] + dt * (S.b[1] + dt * (S.b[2] + dt * S.b[3]));
    const double sn = sin(theta), cs = cos(theta);
    const double theta_dot = S.b[1] + dt * (2.0 * S.b[2] + dt * 3.0 * S.b[3]);
    double rd[9];
    for (int e = 0; e < 9; ++e) {
        const double a = fma(dt, S.k[0][e], S.m[0][e]);
        const double b = fma(dt, S.k[1][e], S.m[1][e]);
        const double c = fma(dt, S.k[2][e], S.m[2][e]);
        out.r[e] = fma(cs, a, fma(sn, b, c));
        const double frozen = fma(cs, S.k[0][e], fma(sn, S.k[1][e], S.k[2][e]));
        rd[e] = fma(theta_dot, fma(-sn, a, cs * b), frozen);
    }
    const double* r = out.r;
    auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    const double wi[3] = {0.5 * (dot(rd + 3, r + 6) - dot(rd + 6, r + 3)),
                          0.5 * (dot(rd + 6, r + 0) - dot(rd + 0, r + 6)),
                          0.5 * (dot(rd + 0, r + 3) - dot(rd + 3, r + 0))};
    // R^T wi
    out.w[0] = r[0] * wi[0] + r[3] * wi[1] + r[6] * wi[2];
    out.w[1] = r[1] * wi[0] + r[4] * wi[1] + r[7] * wi[2];
    out.w[2] = r[2] * wi[0] + r[5] * wi[1] + r[8] * wi[2];
}

// GCRS -> ITRS and back, in the reference's FMA forms (authority.rs:251-272).
BQP_HD void to_itrs(const double* r, const double* v, double* o) {
    o[0] = fma(r[0], v[0], fma(r[1], v[1], r[2] * v[2]));
    o[1] = fma(r[3], v[0], fma(r[4], v[1], r[5] * v[2]));
    o[2] = fma(r[6], v[0], fma(r[7], v[1], r[8] * v[2]));
}
BQP_HD void to_gcrs(const double* r, const double* v, double* o) {
    o[0] = fma(r[0], v[0], fma(r[3], v[1], r[6] * v[2]));
    o[1] = fma(r[1], v[0], fma(r[4], v[1], r[7] * v[2]));
    o[2] = fma(r[2], v[0], fma(r[5], v[1], r[8] * v[2]));
}

// ------------------------------------------------------------ time scales
// TAI - UTC in the integer-leap era (1972-01-01 on), by UTC MJD.  The dates
// are the IERS Bulletin C leap seconds; each entry is the MJD from which the
// count holds (10 s from 1972-01-01, one more at each entry after it).
constexpr int kLeapEntries = 28;
#define BQP_FT_LEAP_MJD                                                                                   \
    {41317, 41499, 41683, 42048, 42413, 42778, 43144, 43509, 43874, 44239, 44786, 45151, 45516, 46247, \
     47161, 47892, 48257, 48804, 49169, 49534, 50083, 50630, 51179, 53736, 54832, 56109, 57204, 57754}

BQP_HD double dat_mjd(int32_t mjd) {
    const int32_t tab[kLeapEntries] = BQP_FT_LEAP_MJD;
    int32_t c = 0;
    for (int q = 0; q < kLeapEntries; ++q) c += mjd >= tab[q] ? 1 : 0;
    return c == 0 ? NAN : (double)(9 + c);
}

BQP_HD double dnint(double a) {
    if (fabs(a) < 0.5) return 0.0;
    return a < 0.0 ? ceil(a - 0.5) : floor(a + 0.5);
}

// Two-part JD -> integer Julian day number and day fraction, with ERFA
// jd2cal's compensated sum (timescale.rs:75-160).  Returns false out of range.
BQP_HD bool jd_split(double dj1, double dj2, int64_t* jd_out, double* fd_out) {
    const double dj = dj1 + dj2;
    if (!(dj >= -68569.5 && dj <= 1e9)) return false;
    double rounded = dnint(dj1);
    const double f1 = dj1 - rounded;
    int64_t jd = (int64_t)rounded;
    rounded = dnint(dj2);
    const double f2 = dj2 - rounded;
    jd += (int64_t)rounded;
    double s = 0.5, cs = 0.0;
    const double fr[2] = {f1, f2};
    for (int i = 0; i < 2; ++i) {
        const double x = fr[i];
        const double t = s + x;
        cs += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
        s = t;
        if (s >= 1.0) {
            jd += 1;
            s -= 1.0;
        }
    }
    double f = s + cs;
    cs = f - s;
    if (f < 0.0) {
        f = s + 1.0;
        cs += (1.0 - f) + s;
        s = f;
        f = s + cs;
        cs = f - s;
        jd -= 1;
    }
    const double eps = 2.220446049250313e-16;
    if ((f - 1.0) >= -eps / 4.0) {
        const double t = s - 1.0;
        cs += (s - t) - 1.0;
        s = t;
        f = s + cs;
        if (-eps / 2.0 < f) {
            jd += 1;
            f = fmax(f, 0.0);
        }
    }
    *jd_out = jd;
    *fd_out = f;
    return true;
}

// UTC (two-part quasi-JD) -> TAI, ERFA utctai in the integer-leap era, where
// TAI - UTC is constant over a day and a day ending in a leap second lasts
// 86,401 s (timescale.rs:440-500).  False before 1972 or out of range.
BQP_HD bool utc_to_tai(double utc1, double utc2, double* tai1, double* tai2) {
    const bool big1 = fabs(utc1) >= fabs(utc2);
    const double u1 = big1 ? utc1 : utc2, u2 = big1 ? utc2 : utc1;
    int64_t jd;
    double fd;
    if (!jd_split(u1, u2, &jd, &fd)) return false;
    const int32_t mjd = (int32_t)(jd - 2400001);  // the civil day holding the instant
    int64_t jdt;
    double fdt;
    if (!jd_split(u1 + 1.5, u2 - fd, &jdt, &fdt)) return false;
    const double dat0 = dat_mjd(mjd);
    const double dat24 = dat_mjd((int32_t)(jdt - 2400001));
    if (!(dat0 == dat0) || !(dat24 == dat24)) return false;
    const double dleap = dat24 - dat0;
    fd = mul_rn(fd, (kDaySec + dleap) / kDaySec);
    double a2 = kDjm0 - u1;
    a2 = add_rn(a2, (double)mjd);
    a2 = add_rn(a2, add_rn(fd, dat0 / kDaySec));
    *tai1 = big1 ? u1 : a2;
    *tai2 = big1 ? a2 : u1;
    return true;
}

// Continuous TAI seconds of a two-part UTC quasi-JD: utctai, then the
// origin removed from the large part (authority.rs:1162-1190).
BQP_HD bool tai_seconds_from_utc_parts(double u1, double u2, double* tai_s) {
    double t1, t2;
    if (!utc_to_tai(u1, u2, &t1, &t2)) return false;
    const double day_part = t1 - kDjm0 - (double)kOriginMjd;
    *tai_s = add_rn(mul_rn(day_part, kDaySec), mul_rn(t2, kDaySec));
    return *tai_s == *tai_s;
}

// The same of a one-part UTC Julian day, split at the civil day's
// noon-based half first (rhs.rs:3090-3093).
BQP_HD bool tai_seconds_from_utc_jd(double jd, double* tai_s) {
    const double big = floor(jd - 0.5) + 0.5;
    return tai_seconds_from_utc_parts(big, jd - big, tai_s);
}

}  // namespace ft
}  // namespace bqp
