// Force-model and element physics shared by the host API and the sm_100a
// kernels (FP64).  Every function here is __host__ __device__ so the host can
// run the same arithmetic for set-up (element conversion of inputs, table
// builds) as the kernels use in the hot loop.
//
// Conventions (dust_transfer/src/lib.rs:1-24 of the reference): km, km/s, s,
// Julian Date (UTC); the inertial frame is the propagator's ECI, the gravity
// field is Earth-fixed; states are [x, y, z, vx, vy, vz].
#pragma once
#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define BQP_HD __host__ __device__ __forceinline__
#else
#define BQP_HD inline
#endif

namespace bqp {

// satpy_core/src/lib.rs:70-113 (reference constants, carried verbatim)
constexpr double kEarthOmega = 7.2921150e-5;        // rad/s
constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kPi = 3.14159265358979323846264338327950;
constexpr double kGmstSec2Rad = (2.0 * kPi) / 86400.0;
constexpr double kGmstLinear = 8640184.812866 + 876600.0 * 3600.0;
constexpr double kGmstConst = 67310.54841;
constexpr double kMu = 398600.4415;                 // km^3/s^2
constexpr double kInvMu = 1.0 / 398600.4415;
constexpr double kReWgs84 = 6378.137;               // km, figure of the Earth
constexpr double kReGravity = 6378.13646;           // km, DIR-R6 reference radius
constexpr double kWgs84F = 1.0 / 298.257223563;
constexpr double kKeplerTol = 1e-12;
constexpr int kKeplerMaxIter = 500;
constexpr double kSecPerDay = 86400.0;
constexpr double kMaxSegmentS = 5400.0;             // integrator.rs:236
constexpr double kRebaseKm = 10.0;                  // types.rs:138
constexpr double kGroundAltitudeKm = 100.0;         // types.rs:140

// ---------------------------------------------------------------- UTC / TAI
// UTC days that start with a new TAI - UTC (IERS Bulletin C): the MJD of
// each day from 1972-01-01 (TAI - UTC = 10 s) on, each later one adding one
// second (the last, 2017-01-01, makes it 37 s).  The day before each later
// entry ends with a leap second and lasts 86,401 s.
#define BQP_LEAP_MJD_LIST                                                                                 \
    {41317, 41499, 41683, 42048, 42413, 42778, 43144, 43509, 43874, 44239, 44786, 45151, 45516, 46247, \
     47161, 47892, 48257, 48804, 49169, 49534, 50083, 50630, 51179, 53736, 54832, 56109, 57204, 57754}
constexpr int kLeapCount = 28;
#ifdef __CUDACC__
__constant__ const int32_t kLeapMjdDev[kLeapCount] = BQP_LEAP_MJD_LIST;
#endif
static const int32_t kLeapMjdHost[kLeapCount] = BQP_LEAP_MJD_LIST;
#ifdef __CUDA_ARCH__
#define BQP_LEAP_MJD kLeapMjdDev
#else
#define BQP_LEAP_MJD kLeapMjdHost
#endif

// Length in SI seconds of UTC day `mjd_day` (an integral MJD).
BQP_HD double utc_day_seconds(double mjd_day) {
    for (int k = 1; k < kLeapCount; ++k)
        if ((double)BQP_LEAP_MJD[k] == mjd_day + 1.0) return 86401.0;
    return 86400.0;
}

// UTC Julian day of the instant t seconds after the epoch jd0 (a UTC Julian
// day): the propagator integrates in continuous (TAI) seconds, and the
// JB2008 drivers, the ephemeris catalogues and the Earth's rotation are
// looked up on UTC (lightyear_odeint_rs/src/rhs.rs:3090-3110, 3264-3300).  UTC
// Julian days of a day that ends in a leap second run over 86,401 s (the
// ERFA convention the reference follows), so the leap second 23:59:60 is day
// fraction 86400/86401.  Where no such day is within a day of the arc this
// is jd0 + t/86400 to the bit; before 1972 it is that always.
BQP_HD double utc_jd_at(double jd0, double t) {
    const double plain = jd0 + t / kSecPerDay;
    const double mjd0 = jd0 - 2400000.5;
    if (!(isfinite(mjd0) && isfinite(t)) || mjd0 < (double)BQP_LEAP_MJD[0]) return plain;
    const double d0 = floor(mjd0), d1 = floor(mjd0 + t / kSecPerDay);
    const double lo = fmin(d0, d1) - 1.0, hi = fmax(d0, d1) + 1.0;
    bool near_leap = false;
    for (int k = 1; k < kLeapCount; ++k) {
        const double last = (double)BQP_LEAP_MJD[k] - 1.0;  // the day that ends in the leap second
        if (last >= lo && last <= hi) near_leap = true;
    }
    if (!near_leap) return plain;
    // walk whole UTC days from the epoch's, in SI seconds (arcs span days;
    // the bound only guarantees an end)
    double d = d0;
    double sec = (mjd0 - d0) * utc_day_seconds(d0) + t;
    for (int it = 0; it < 100000; ++it) {
        if (sec < 0.0) {
            d -= 1.0;
            sec += utc_day_seconds(d);
        } else if (sec >= utc_day_seconds(d)) {
            sec -= utc_day_seconds(d);
            d += 1.0;
        } else {
            break;
        }
    }
    return (2400000.5 + d) + sec / utc_day_seconds(d);
}

BQP_HD double mod2pi(double a) {
    if (!isfinite(a)) return NAN;
    double x = fmod(a, kTwoPi);
    if (x < 0.0) x += kTwoPi;
    if (x >= kTwoPi) x -= kTwoPi;
    return x == 0.0 ? 0.0 : x;
}

BQP_HD double clamp_ecc(double e) {
    if (!isfinite(e) || e <= 0.0) return 0.0;
    if (e >= 1.0) {
        double c = 1.0 - 10.0 * kKeplerTol;
        return c > 0.0 ? c : 0.0;
    }
    return e;
}

// Greenwich mean sidereal angle of a UTC Julian Date (satpy lib.rs:905-912).
BQP_HD double gmst_rad(double jd) {
    double t = (jd - 2451545.0) / 36525.0;
    double sec = fma(fma(fma(-6.2e-6, t, 0.093104), t, kGmstLinear), t, kGmstConst);
    return mod2pi(sec * kGmstSec2Rad);
}

// ----------------------------------------------------------------- elements
// Equinoctial elements [a, h, k, p, q, L] (retrograde-singular form) from an
// ECI state (satpy lib.rs:1879-2012).  Returns false (and NaNs) for an
// unbound or degenerate orbit.
BQP_HD bool eci_to_equinoctial(const double* st, double* out) {
    double rx = st[0], ry = st[1], rz = st[2], vx = st[3], vy = st[4], vz = st[5];
    double rn = sqrt(rx * rx + ry * ry + rz * rz);
    double vn = sqrt(vx * vx + vy * vy + vz * vz);
    double inv_r = 1.0 / rn;
    double energy = fma(0.5, vn * vn, -kMu * inv_r);
    bool ok = energy < -1e-12;
    double hx = ry * vz - rz * vy, hy = rz * vx - rx * vz, hz = rx * vy - ry * vx;
    double hn = sqrt(hx * hx + hy * hy + hz * hz);
    double inv_h = 1.0 / hn;
    double tx = vy * hz - vz * hy, ty = vz * hx - vx * hz, tz = vx * hy - vy * hx;
    double ex = fma(tx, kInvMu, -rx * inv_r);
    double ey = fma(ty, kInvMu, -ry * inv_r);
    double ez = fma(tz, kInvMu, -rz * inv_r);
    double emag = sqrt(ex * ex + ey * ey + ez * ez);
    double es = (!isfinite(emag) || emag <= 0.0) ? 0.0 : (emag >= 1.0 ? 1.0 - 1e-11 : emag);
    double a = -kMu / (2.0 * energy);
    ok = ok && a > 0.0;
    double nz = hz * inv_h;
    double dh = 1.0 + nz;
    double hc = fabs(dh) < 1e-12 ? 0.0 : (1.0 - nz) / dh;
    double p = (1.0 + hc) * hx * inv_h * 0.5;
    double q = -(1.0 + hc) * hy * inv_h * 0.5;
    double p2 = p * p, q2 = q * q, tpq = 2.0 * p * q;
    double coef = 1.0 / fma(p2, 1.0, fma(q2, 1.0, 1.0));
    double xh0 = coef * fma(q2, 1.0, 1.0 - p2), xh1 = coef * tpq, xh2 = coef * (-2.0 * p);
    double yh0 = coef * tpq, yh1 = coef * fma(p2, 1.0, 1.0 - q2), yh2 = coef * (2.0 * q);
    double hv = yh0 * ex + yh1 * ey + yh2 * ez;
    double kv = xh0 * ex + xh1 * ey + xh2 * ez;
    double xd = xh0 * vx + xh1 * vy + xh2 * vz;
    double yd = yh0 * vx + yh1 * vy + yh2 * vz;
    double sqrt_ma = sqrt(kMu * a);
    double coef2 = rn / sqrt_ma;
    double sq = sqrt(fmax(1.0 - es * es, 0.0));
    double ds = 1.0 + sq;
    double sds = fabs(ds) < 1e-12 ? (ds >= 0.0 ? 1e-12 : -1e-12) : ds;
    double coef3 = (rn * (1.0 / a) - 1.0) / sds;
    double sf = fma(-xd, coef2, -hv * coef3);
    double cf = fma(yd, coef2, -kv * coef3);
    double fa = atan2(sf, cf);
    double sfa, cfa;
    sincos(fa, &sfa, &cfa);
    double lam = fa + fma(hv, cfa, -kv * sfa);
    if (isfinite(lam)) {
        lam = fmod(lam, kTwoPi);
        if (lam < 0.0) lam += kTwoPi;
        if (lam >= kTwoPi) lam -= kTwoPi;
    } else {
        lam = NAN;
    }
    out[0] = a; out[1] = hv; out[2] = kv; out[3] = p; out[4] = q; out[5] = lam;
    ok = ok && isfinite(a) && isfinite(hv) && isfinite(kv) && isfinite(p) && isfinite(q) &&
         isfinite(lam);
    if (!ok)
        for (int i = 0; i < 6; ++i) out[i] = NAN;
    return ok;
}

// Analytic two-body baseline from equinoctial elements (the Encke reference
// orbit; satpy lib.rs:2191-2374): element-only terms are hoisted here, the
// per-time half solves the equinoctial Kepler equation F + h cosF - k sinF = L
// by Halley-type iteration.
struct Baseline {
    double a, h, k, n, ecoef, L0;
    double xh0, xh1, xh2, yh0, yh1, yh2;
    int ok;
};

BQP_HD Baseline baseline_new(const double* e) {
    Baseline b;
    b.ok = 0;
    double a = e[0], h = e[1], k = e[2], p = e[3], q = e[4];
    b.a = a; b.h = h; b.k = k; b.L0 = e[5];
    double er = sqrt(fma(h, h, k * k));
    double ecc = clamp_ecc(er);
    double p2 = p * p, q2 = q * q;
    double coef = 1.0 / fma(p2, 1.0, fma(q2, 1.0, 1.0));
    b.n = sqrt(kMu / (a * a * a));
    b.ecoef = 1.0 + sqrt(fmax(fma(ecc, -ecc, 1.0), 0.0));
    b.xh0 = coef * fma(q2, 1.0, 1.0 - p2);
    b.xh1 = coef * (2.0 * p * q);
    b.xh2 = coef * (-2.0 * p);
    b.yh0 = coef * (2.0 * p * q);
    b.yh1 = coef * fma(p2, 1.0, 1.0 - q2);
    b.yh2 = coef * (2.0 * q);
    b.ok = (a > 0.0 && er < 1.0) ? 1 : 0;
    return b;
}

// State on the baseline orbit `tof` seconds after the elements' epoch.
// Returns false (out[0] = NaN) if the baseline is invalid or the iteration
// does not converge.
BQP_HD bool baseline_state(const Baseline& b, double tof, double* out) {
    if (!b.ok) {
        for (int i = 0; i < 6; ++i) out[i] = NAN;
        return false;
    }
    double L = mod2pi(b.L0 + b.n * tof);
    double F = L;
    double sF, cF;
    sincos(F, &sF, &cF);
    int it = 0;
    for (; it < kKeplerMaxIter; ++it) {
        double at = b.h * cF - b.k * sF;
        double bt = b.h * sF + b.k * cF;
        double f0 = F + at - L;
        double f1 = 1.0 - bt;
        double d1 = -f0 / f1;
        double d2 = -f0 / (f1 + 0.5 * d1 * (-at));
        double d3 = -f0 / (f1 + 0.5 * d2 * (-at) + (1.0 / 6.0) * d2 * d2 * bt);
        F = F + d3;
        if (fabs(d3) < kKeplerTol) break;
        double sd, cd;
        sincos(d3, &sd, &cd);
        double sn = fma(sF, cd, cF * sd);
        cF = fma(cF, cd, -sF * sd);
        sF = sn;
    }
    if (it == kKeplerMaxIter) {
        for (int i = 0; i < 6; ++i) out[i] = NAN;
        return false;
    }
    double cl = (L - F) / b.ecoef;
    double X = b.a * (cF - b.k - b.h * cl);
    double Y = b.a * (sF - b.h + b.k * cl);
    double px = b.xh0 * X + b.yh0 * Y;
    double py = b.xh1 * X + b.yh1 * Y;
    double pz = b.xh2 * X + b.yh2 * Y;
    double rn = sqrt(fma(px, px, fma(py, py, pz * pz)));
    double Fd = b.a * b.n / rn;
    double c3 = (b.n - Fd) / b.ecoef;
    double Xd = b.a * fma(-Fd, sF, -b.h * c3);
    double Yd = b.a * fma(Fd, cF, b.k * c3);
    out[0] = px; out[1] = py; out[2] = pz;
    out[3] = b.xh0 * Xd + b.yh0 * Yd;
    out[4] = b.xh1 * Xd + b.yh1 * Yd;
    out[5] = b.xh2 * Xd + b.yh2 * Yd;
    return true;
}

BQP_HD bool equinoctial_to_eci(const double* e, double tof, double* out) {
    Baseline b = baseline_new(e);
    return baseline_state(b, tof, out);
}

// ---------------------------------------------------------------- ephemeris
// Low-precision analytic Sun and Moon positions (Montenbruck & Gill,
// "Satellite Orbits", 2000, section 3.3.2), J2000 equator/equinox, km.  The
// reference reads precomputed catalogues (precomputed_ephem.rs); with a
// catalogue set (EphemTable below) the kernels read it the same way, and
// these series stand in for it otherwise.
constexpr double kDeg = kPi / 180.0;
constexpr double kArcsec = kDeg / 3600.0;
constexpr double kObliquity = 23.43929111 * kDeg;

BQP_HD void sun_position(double jd, double* out) {
    double T = (jd - 2451545.0) / 36525.0;
    double M = mod2pi((357.5256 + 35999.049 * T) * kDeg);
    double sM, cM;
    sincos(M, &sM, &cM);
    double s2M = 2.0 * sM * cM, c2M = cM * cM - sM * sM;
    double lam = 282.9400 * kDeg + M + 6892.0 * kArcsec * sM + 72.0 * kArcsec * s2M;
    double r = (149.619 - 2.499 * cM - 0.021 * c2M) * 1e6;
    double sl, cl;
    sincos(lam, &sl, &cl);
    const double ce = 0.9174820620768958, se = 0.3977771559141214;  // cos, sin of 23.43929111 deg
    out[0] = r * cl;
    out[1] = ce * (r * sl);
    out[2] = se * (r * sl);
}

// (sin, cos) pair with angle-addition helpers: the Moon series below needs
// the sines and cosines of ~30 integer combinations of four fundamental
// arguments; they are built from the four sincos pairs instead of one
// transcendental call each.
struct SC {
    double s, c;
};
BQP_HD SC sc_add(SC a, SC b) { return {fma(a.s, b.c, a.c * b.s), fma(a.c, b.c, -(a.s * b.s))}; }
BQP_HD SC sc_sub(SC a, SC b) { return {fma(a.s, b.c, -(a.c * b.s)), fma(a.c, b.c, a.s * b.s)}; }
BQP_HD SC sc_dbl(SC a) { return {2.0 * a.s * a.c, fma(a.c, a.c, -(a.s * a.s))}; }
BQP_HD SC sc_of(double x) {
    SC r;
    sincos(x, &r.s, &r.c);
    return r;
}

BQP_HD void moon_position(double jd, double* out) {
    double T = (jd - 2451545.0) / 36525.0;
    const double L0 = mod2pi((218.31617 + 481267.88088 * T - 1.3972 * T) * kDeg);
    const SC l = sc_of(mod2pi((134.96292 + 477198.86753 * T) * kDeg));
    const SC lp = sc_of(mod2pi((357.52543 + 35999.04944 * T) * kDeg));
    const double Fang = mod2pi((93.27283 + 483202.01873 * T) * kDeg);
    const SC F = sc_of(Fang);
    const SC D = sc_of(mod2pi((297.85027 + 445267.11135 * T) * kDeg));
    const SC l2 = sc_dbl(l), D2 = sc_dbl(D), F2 = sc_dbl(F);
    const SC l_2D = sc_sub(l, D2);          // l - 2D
    const SC l2_2D = sc_sub(l2, D2);        // 2l - 2D
    const SC llp_2D = sc_add(l_2D, lp);     // l + l' - 2D
    const SC lp2D = sc_add(l, D2);          // l + 2D
    const SC lp_2D = sc_sub(lp, D2);        // l' - 2D
    const SC l_lp = sc_sub(l, lp);          // l - l'
    const SC llp = sc_add(l, lp);           // l + l'
    const SC F2_2D = sc_sub(F2, D2);        // 2F - 2D
    const SC F_2D = sc_sub(F, D2);          // F - 2D
    const double dlam = 22640.0 * l.s + 769.0 * l2.s - 4586.0 * l_2D.s + 2370.0 * D2.s - 668.0 * lp.s -
                        412.0 * F2.s - 212.0 * l2_2D.s - 206.0 * llp_2D.s + 192.0 * lp2D.s - 165.0 * lp_2D.s +
                        148.0 * l_lp.s - 125.0 * D.s - 110.0 * llp.s - 55.0 * F2_2D.s;
    const double lam = L0 + dlam * kArcsec;
    // argument of the main latitude term: F + (lam - L0) + (412 sin 2F + 541 sin l')"
    const double argF = Fang + dlam * kArcsec + (412.0 * F2.s + 541.0 * lp.s) * kArcsec;
    const SC lF_2D = sc_add(l_2D, F);       // l + F - 2D
    const SC mlF_2D = sc_sub(F_2D, l);      // -l + F - 2D
    const SC m2lF = sc_sub(F, l2);          // -2l + F
    const SC lpF_2D = sc_add(F_2D, lp);     // l' + F - 2D
    const SC mlF = sc_sub(F, l);            // -l + F
    const SC mlpF_2D = sc_sub(F_2D, lp);    // -l' + F - 2D
    double beta = 18520.0 * sin(argF) - 526.0 * F_2D.s + 44.0 * lF_2D.s - 31.0 * mlF_2D.s - 25.0 * m2lF.s -
                  23.0 * lpF_2D.s + 21.0 * mlF.s + 11.0 * mlpF_2D.s;
    beta *= kArcsec;
    const SC D2_l = sc_sub(D2, l);          // 2D - l
    const double r = 385000.0 - 20905.0 * l.c - 3699.0 * D2_l.c - 2956.0 * D2.c - 570.0 * l2.c + 246.0 * l2_2D.c -
                     205.0 * lp_2D.c - 171.0 * lp2D.c - 152.0 * llp_2D.c;
    double sb, cb, sl, cl;
    sincos(beta, &sb, &cb);
    sincos(lam, &sl, &cl);
    const double xe = r * cb * cl, ye = r * cb * sl, ze = r * sb;
    const double ce = 0.9174820620768958, se = 0.3977771559141214;
    out[0] = xe;
    out[1] = ce * ye - se * ze;
    out[2] = se * ye + ce * ze;
}

// Point-mass third body in the normalised form of rhs.rs:1326-1354.
// Precomputed Sun / Moon catalogue as the kernels read it: samples of
// Earth-centred ICRS positions (km) every dt days from jd_start (UTC Julian
// days).  n == 0: no catalogue, the analytic series apply.
struct EphemTable {
    const double* pos;  // [n][3]
    double jd_start, jd_end, dt, inv_dt;  // jd_end = jd_start + (n - 1) dt, inv_dt = 1 / dt
    int64_t n;
};

// a (1 - f) + b f, as the reference rounds it (no contraction on the device)
BQP_HD double eph_lerp(double a, double b, double f) {
#ifdef __CUDA_ARCH__
    return __dadd_rn(__dmul_rn(a, __dsub_rn(1.0, f)), __dmul_rn(b, f));
#else
    return a * (1.0 - f) + b * f;
#endif
}

BQP_HD void eph_interp(const EphemTable& E, int64_t i, double f, double* out) {
    for (int k = 0; k < 3; ++k) out[k] = eph_lerp(E.pos[3 * i + k], E.pos[3 * (i + 1) + k], f);
}

BQP_HD void eph_sample(const EphemTable& E, int64_t i, double* out) {
    for (int k = 0; k < 3; ++k) out[k] = E.pos[3 * i + k];
}

// Position at a UTC Julian day (precomputed_ephem.rs:1092-1131 linear
// interpolation on the grid; outside it, only JD roundoff of 2 eps at an end
// is clamped, rhs.rs:2996-3018); NaN otherwise.
BQP_HD void ephem_position(const EphemTable& E, double jd, double* out) {
    constexpr double kEps = 2.220446049250313e-16;
    if (isfinite(jd)) {
        if (E.n == 1) {
            if (fabs(jd - E.jd_start) <= kEps) return eph_sample(E, 0, out);
        } else {
            const double fi = (jd - E.jd_start) * E.inv_dt;
            const double last = (double)(E.n - 1);
            if (fi >= 0.0 && fi <= last) {
                if (fi >= last) return eph_sample(E, E.n - 1, out);
                const int64_t i = (int64_t)fi;
                return eph_interp(E, i, fi - (double)i, out);
            }
        }
        const double cl = fmin(fmax(jd, E.jd_start), E.jd_end);
        const double tol = 2.0 * kEps * fmax(fabs(jd), fmax(fabs(E.jd_start), fabs(E.jd_end)));
        if (fabs(jd - cl) <= tol) {
            if (E.n < 2 || cl <= E.jd_start) return eph_sample(E, 0, out);
            if (cl >= E.jd_end) return eph_sample(E, E.n - 1, out);
            const double fi = (cl - E.jd_start) * E.inv_dt;
            const int64_t i = (int64_t)fi;
            if (i + 1 < E.n) return eph_interp(E, i, fi - (double)i, out);
            // 1/dt rounded the index onto the last sample: the reference finds
            // no next sample there and answers the origin
            out[0] = out[1] = out[2] = 0.0;
            return;
        }
    }
    out[0] = out[1] = out[2] = NAN;
}

// Sun or Moon: the catalogue when one is set, else the analytic series.
BQP_HD void sun_at(const EphemTable& E, double jd, double* out) {
    if (E.n > 0) ephem_position(E, jd, out);
    else sun_position(jd, out);
}
BQP_HD void moon_at(const EphemTable& E, double jd, double* out) {
    if (E.n > 0) ephem_position(E, jd, out);
    else moon_position(jd, out);
}

BQP_HD void third_body(const double* sat, const double* body, double mu_body, double* acc) {
    double d2 = body[0] * body[0] + body[1] * body[1] + body[2] * body[2];
    if (d2 == 0.0) return;
    double inv_d = 1.0 / sqrt(d2);
    double mu_coef = mu_body * (inv_d * inv_d);
    double bn0 = body[0] * inv_d, bn1 = body[1] * inv_d, bn2 = body[2] * inv_d;
    double r0 = bn0 - sat[0] * inv_d, r1 = bn1 - sat[1] * inv_d, r2 = bn2 - sat[2] * inv_d;
    double rd2 = fma(r0, r0, fma(r1, r1, r2 * r2));
    if (rd2 == 0.0) return;
    double inv3 = 1.0 / (rd2 * sqrt(rd2));
    acc[0] += mu_coef * (r0 * inv3 - bn0);
    acc[1] += mu_coef * (r1 * inv3 - bn1);
    acc[2] += mu_coef * (r2 * inv3 - bn2);
}

// ------------------------------------------ solar radiation pressure, shadow
constexpr double kAuKm = 149597870.7;
constexpr double kPSun = 4.56e-6;  // N/m^2 at 1 AU (types.rs:459)

// Binary shadow cylinder of the Earth along the Sun direction
// (eclipse.rs:189-262): *shadow 1 behind the Earth inside the cylinder,
// else 0; *margin the distance to the boundary (the nearer of the axial and
// radial distances in shadow).  False on invalid geometry.
BQP_HD bool shadow_cylinder(const double* sat, const double* sun, double earth_radius, int* shadow,
                            double* margin) {
    for (int i = 0; i < 3; ++i)
        if (!isfinite(sat[i]) || !isfinite(sun[i])) return false;
    if (!(isfinite(earth_radius) && earth_radius > 0.0)) return false;
    const double sun_sq = sun[0] * sun[0] + sun[1] * sun[1] + sun[2] * sun[2];
    if (!(isfinite(sun_sq) && sun_sq > 0.0)) return false;
    const double inv = 1.0 / sqrt(sun_sq);
    const double u0 = sun[0] * inv, u1 = sun[1] * inv, u2 = sun[2] * inv;
    const double axial = fma(sat[0], u0, fma(sat[1], u1, sat[2] * u2));
    const double q0 = sat[0] - axial * u0, q1 = sat[1] - axial * u1, q2 = sat[2] - axial * u2;
    const double rad_sq = fma(q0, q0, fma(q1, q1, q2 * q2));
    const double r_sq = earth_radius * earth_radius;
    if (!(isfinite(axial) && isfinite(rad_sq) && isfinite(r_sq))) return false;
    const double rd = sqrt(rad_sq);
    const double signed_margin = (rad_sq - r_sq) / (rd + earth_radius);
    double m;
    if (axial < 0.0 && rad_sq < r_sq) {
        *shadow = 1;
        m = fmin(-axial, -signed_margin);
    } else {
        *shadow = 0;
        const bool a = axial >= 0.0, b = rad_sq >= r_sq;
        m = a && b ? fmax(axial, signed_margin) : (a ? axial : (b ? signed_margin : 0.0));
    }
    if (!(isfinite(m) && m >= 0.0)) return false;
    *margin = m;
    return true;
}

// Cannonball solar radiation pressure (rhs.rs:1269-1310) added into acc
// (km/s^2): p_sun cr A/m (AU/d)^2 away from the Sun, none in shadow.
BQP_HD void srp_accel(const double* sat, const double* sun, double p_sun, double cr, double am, int shadow,
                      double* acc) {
    if (cr == 0.0 || am == 0.0 || p_sun == 0.0) return;
    if (!isfinite(sat[0]) || !isfinite(sat[1]) || !isfinite(sat[2])) {
        acc[0] = acc[1] = acc[2] = NAN;
        return;
    }
    if (shadow) return;
    const double rx = sun[0] - sat[0], ry = sun[1] - sat[1], rz = sun[2] - sat[2];
    const double d2 = fma(rx, rx, fma(ry, ry, rz * rz));
    if (!(isfinite(d2) && d2 > 0.0)) {
        acc[0] = acc[1] = acc[2] = NAN;
        return;
    }
    const double inv = 1.0 / sqrt(d2);
    const double a = p_sun * cr * am * ((kAuKm * kAuKm) / d2) * 0.001;
    acc[0] += -a * rx * inv;
    acc[1] += -a * ry * inv;
    acc[2] += -a * rz * inv;
}

// Battin's f(q) form of the Encke central-body difference (rhs.rs:1071-1104):
// mu (r_b/|r_b|^3 - r_p/|r_p|^3) = mu/|r_p|^3 (f(q) r_b - dr).
BQP_HD void battin(const double* rb, const double* dr, double rp2, double rp, double* acc) {
    double rb2 = fma(rb[0], rb[0], fma(rb[1], rb[1], rb[2] * rb[2]));
    if (!(rb2 > 0.0 && rp2 > 0.0)) return;
    double ddot = fma(dr[0], rb[0], fma(dr[1], rb[1], dr[2] * rb[2]));
    double dsq = fma(dr[0], dr[0], fma(dr[1], dr[1], dr[2] * dr[2]));
    double q = (dsq + 2.0 * ddot) / rb2;
    double q1 = 1.0 + q;
    double fq = q * (3.0 + q * (3.0 + q)) / (1.0 + q1 * sqrt(q1));
    double k = kMu * (1.0 / (rp2 * rp));
    acc[0] += k * fma(fq, rb[0], -dr[0]);
    acc[1] += k * fma(fq, rb[1], -dr[1]);
    acc[2] += k * fma(fq, rb[2], -dr[2]);
}

// WGS84 geodetic altitude of an Earth-fixed position, one Bowring step
// (rhs.rs:160-186).
BQP_HD double geodetic_altitude_km(double x, double y, double z, double a) {
    const double omf = 1.0 - kWgs84F;
    const double e2 = kWgs84F * (2.0 - kWgs84F);
    const double ep2 = e2 / (omf * omf);
    double req = sqrt(fma(x, x, y * y));
    if (req == 0.0) return fabs(z) - a * omf;
    double b = a * omf;
    double tn = z * a, td = req * b;
    double tr = sqrt(fma(tn, tn, td * td));
    double st = tn / tr, ct = td / tr;
    double ln = z + ep2 * b * st * st * st;
    double ld = req - e2 * a * ct * ct * ct;
    double lr = sqrt(fma(ln, ln, ld * ld));
    double sl = ln / lr, cl = ld / lr;
    double om = 1.0 - e2 * sl * sl;
    double nrad = a / sqrt(om);
    return req * cl + z * sl - nrad * om;
}

}  // namespace bqp
