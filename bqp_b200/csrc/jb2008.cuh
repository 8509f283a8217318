// Jacchia-Bowman 2008 thermospheric density (Bowman et al., AIAA 2008-6438),
// in the form Orekit 13.1.2 implements and the reference adapts
// (jb_rs/src/jb2008.rs, "exact" quadrature profile): exospheric temperature
// from the solar indices, the local-temperature profile, Boole-rule
// integration of the barometric / diffusion equations from 90 km through 105
// and 500 km, six species, the semiannual and seasonal-latitudinal
// corrections and the high-altitude density factor.  The coefficient tables
// are the published model's (they must match it to reproduce the model).
//
// Host and device share this code.  FP64 throughout; the quadrature node
// count depends only on altitude, so a warp whose trajectories share an
// altitude band walks the same loop trip counts.
#pragma once
#include "physics.cuh"

namespace bqp {
namespace jb {

// Each table exists twice: in constant memory for the kernels and as a plain
// host array for host-side callers; JBT() picks the copy of the current pass.
#ifdef __CUDACC__
#define BQP_JB_TABLE(name, n, ...)                 \
    __constant__ const double name##_dev[n] = __VA_ARGS__; \
    static const double name##_host[n] = __VA_ARGS__;
#else
#define BQP_JB_TABLE(name, n, ...) static const double name##_host[n] = __VA_ARGS__;
#endif
#ifdef __CUDA_ARCH__
#define JBT(name) name##_dev
#else
#define JBT(name) name##_host
#endif

BQP_JB_TABLE(kAmw, 6, {28.0134, 31.9988, 15.9994, 39.9480, 4.0026, 1.00797})
BQP_JB_TABLE(kFrac, 4, {0.78110, 0.20955, 9.3400e-3, 1.2890e-5})
BQP_JB_TABLE(kBdt, 19, {-4.57512297, -5.12114909, -69.3003609, 203.716701, 703.316291,
                                -1943.49234, 1106.51308, -174.378996, 1885.94601, -7093.71517,
                                9224.54523, -3845.08073, -6.45841789, 40.9703319, -482.006560,
                                1818.70931, -2373.89204, 996.703815, 36.1416936})
BQP_JB_TABLE(kCdt, 23, {-15.5986211, -5.12114909, -69.3003609, 203.716701, 703.316291,
                                -1943.49234, 1106.51308, -220.835117, 1432.56989, -3184.81844,
                                3289.81513, -1353.32119, 19.9956489, -12.7093998, 21.2825156,
                                -2.75555432, 11.0234982, 148.881951, -751.640284, 637.876542,
                                12.7093998, -21.2825156, 2.75555432})
BQP_JB_TABLE(kCxamb, 7, {28.15204, -8.5586e-2, 1.2840e-4, -1.0056e-5, -1.0210e-5,
                                 1.5044e-6, 9.9826e-8})
BQP_JB_TABLE(kCht, 4, {0.22, -0.20e-2, 0.115e-2, -0.211e-5})
BQP_JB_TABLE(kFzm, 5, {0.2689, -0.01176, 0.02782, -0.02782, 0.0003470})
BQP_JB_TABLE(kGtm, 10, {-0.3633, 0.08506, 0.2401, -0.1897, -0.2554,
                                -0.01790, 0.0005650, -0.0006407, -0.003418, -0.001252})

constexpr double kAvogadro = 6.02257e26;
constexpr double kRstar = 8.31432;
constexpr double kW0 = 0.311111111111111, kW1 = 1.422222222222222, kW2 = 0.533333333333333;
constexpr double kEarthR = 6356.766;  // US Standard Atmosphere geopotential radius
constexpr double kG0 = 9.80665;
constexpr double kLnStepLower = 0.010, kLnStepMiddle = 0.025, kLnStepUpper = 0.075;
constexpr double kLn10 = 2.302585092994045684;

// Error codes returned as negative densities.
constexpr double kErrNonFinite = -1.0, kErrAltitude = -2.0, kErrAngle = -3.0, kErrIndex = -4.0,
                 kErrDomain = -5.0;

struct Drivers {
    double f10, f10b, s10, s10b, m10, m10b, y10, y10b, dtc;  // dtc: temperature correction, K
};

// Space-weather tables as the kernels read them: the daily SOLFSMY indices
// and the hourly DTCFILE temperature corrections (jb_rs/src/drivers.rs).
// n_solar == 0: no tables, the fixed drivers apply.
struct DriverTable {
    const double* solar;  // [n_solar][8]: F10, F81c, S10, S81c, M10, M81c, Y10, Y81c
    const int32_t* dtc;   // [n_dtc][24] hourly dTc, K
    double first_jd;      // Julian day number (the row's noon key) of solar row 0
    int32_t n_solar;
    int32_t n_dtc;
    int32_t dtc_first;    // solar row of DTC row 0; DTC days are consecutive SOLFSMY days
};

// Drivers at a UTC Julian day (drivers.rs:559-580, 631-780): F10/S10 and
// their 81-day means from the day before, M10 from two days before, Y10 from
// five; dTc interpolated between the hourly values (the next day's first
// value in the last hour) and rounded half up, with SET's 1e-7 day bias.
// The instant goes through MJD and back, as the reference's lookup entry
// does.  False where the tables do not cover the instant.
BQP_HD bool lookup_drivers(const DriverTable& T, double jd_in, Drivers* d) {
    if (T.n_solar <= 0 || !isfinite(jd_in)) return false;
    const double jd = (jd_in - 2400000.5) + 2400000.5;
    const double day_jd = floor(jd + 0.5);
    const double off = day_jd - T.first_jd;
    if (!(off >= 0.0 && off < (double)T.n_solar)) return false;
    const int i = (int)off;
    if (i < 5) return false;  // the 5-day Y10 lag reaches before the table
    const double frac = jd - (day_jd - 0.5);
    if (!(frac >= 0.0 && frac < 1.0)) return false;
    const int r = i - T.dtc_first;
    if (r < 0 || r >= T.n_dtc) return false;
    const double hour = fmin((frac + 0.0000001) * 24.0, 23.999999999999996);
    const double lh = floor(hour);
    const int h0 = (int)lh;
    const double fraction = hour - lh;
    double upper;
    if (h0 == 23 && fraction > 0.0) {
        if (r + 1 >= T.n_dtc) return false;
        upper = (double)T.dtc[(size_t)(r + 1) * 24];
    } else {
        upper = (double)T.dtc[(size_t)r * 24 + (h0 + 1 < 23 ? h0 + 1 : 23)];
    }
    const double lower = (double)T.dtc[(size_t)r * 24 + h0];
#ifdef __CUDA_ARCH__
    const double v = trunc(__dadd_rn(__dadd_rn(lower, __dmul_rn(fraction, upper - lower)), 0.5));
#else
    const double v = trunc((lower + fraction * (upper - lower)) + 0.5);
#endif
    if (!(v >= -2147483648.0 && v <= 2147483647.0)) return false;
    const double* a = T.solar + (size_t)(i - 1) * 8;
    const double* m = T.solar + (size_t)(i - 2) * 8;
    const double* y = T.solar + (size_t)(i - 5) * 8;
    *d = Drivers{a[0], a[1], a[2], a[3], m[4], m[5], y[6], y[7], v};
    return true;
}

// Fixed-node sweeps as functions of the exospheric temperature.  Above 105
// km the lower Boole sweep (90 -> 105 km) always walks the same 16 intervals,
// and above 500 km the middle sweep (105 -> 500 km) the same 63: their node
// altitudes are constant and their sums depend only on T_inf (through the
// temperature profile tc).  The host fits each sum with a Chebyshev series in
// T_inf (build_jb_fit, 64 terms, checked against the quadrature to ~1e-15
// relative over [lo, hi]); the device evaluates it by Clenshaw's recurrence
// instead of walking ~320 nodes.  Outside [lo, hi], or below 105 / 500 km,
// the quadrature runs as before.
constexpr int kFitTerms = 64;
struct JbFit {
    int32_t valid;
    int32_t terms;
    double lo, hi;
    double low[kFitTerms];  // lower-sweep sum
    double mid[kFitTerms];  // middle-sweep sum
    double low_z, low_zend, low_mb2, low_gravl;  // last node of the lower sweep
    double mid_z, mid_zend, mid_gravl;           // last node of the middle sweep
};

// Sweeps whose node altitudes move with the state's altitude, fitted in two
// variables.  Each sweep's interval count n is a step function of altitude
// (n = 1 + floor(ln(ratio) / step)); inside one n the Boole sum is a smooth
// function of the log-ratio and of T_inf, so each (family, n) gets a
// Chebyshev series in both (kFit2A x kFit2T terms, T_inf over the context's
// own range).  Families:
//   mid:    105 km -> altitude, 105 < alt < 500 km (after the lower fit)
//   uplow:  altitude -> 500 km (the hydrogen anchor), 105 < alt < 500 km
//   uphigh: 500 km -> altitude, 500 < alt <= 2500 km (after the middle fit)
// The node positions themselves are recomputed exactly (the same chain of
// multiplications the quadrature walks); only the sum comes from the fit.
// The host builds and checks every family (build_jb_fit2); a family that
// misses its error bound is switched off and the quadrature runs.
constexpr int kFit2A = 12, kFit2T = 20;
constexpr int kFit2Mid = 64, kFit2UpLow = 64, kFit2UpHigh = 24;
struct JbFit2 {
    int32_t valid_mid, valid_uplow, valid_uphigh, pad;
    double tlo, thi;  // T_inf domain
    // per segment (index n - 1): the log-ratio range the altitudes of the
    // family reach inside it, and the series over that range
    double mid_rng[kFit2Mid][2], uplow_rng[kFit2UpLow][2], uphigh_rng[kFit2UpHigh][2];
    // intervals [first, last] whose nodes can cross the 125 km break of the
    // temperature profile inside the segment: left out of the series and
    // walked exactly ([-1, -1]: none)
    int32_t mid_ex[kFit2Mid][2], uplow_ex[kFit2UpLow][2], uphigh_ex[kFit2UpHigh][2];
    double mid[kFit2Mid][kFit2A][kFit2T];
    double uplow[kFit2UpLow][kFit2A][kFit2T];
    double uphigh[kFit2UpHigh][kFit2A][kFit2T];
};

BQP_HD double fit2_x(const double* rng, double al) { return (2.0 * al - (rng[1] + rng[0])) / (rng[1] - rng[0]); }

// 2-D Chebyshev series c[ka][kt] at (xa, xt), both in [-1, 1].
BQP_HD double cheb2_eval(const double* c, double xa, double xt) {
    double a1 = 0.0, a2 = 0.0;
    for (int ka = kFit2A - 1; ka >= 0; --ka) {
        const double* r = c + ka * kFit2T;
        double b1 = 0.0, b2 = 0.0;
        for (int j = kFit2T - 1; j >= 1; --j) {
            const double tmp = fma(2.0 * xt, b1, -b2) + r[j];
            b2 = b1;
            b1 = tmp;
        }
        const double v = fma(xt, b1, -b2) + r[0];
        if (ka == 0) return fma(xa, a1, -a2) + v;
        const double tmp = fma(2.0 * xa, a1, -a2) + v;
        a2 = a1;
        a1 = tmp;
    }
    return 0.0;
}

// Final node altitude and interval end of an n-interval log-spaced chain
// from zend_start with ratio zr: the same operations the quadrature walks.
BQP_HD void sweep_chain(double zend_start, double zr, int n, double* z_last, double* zend_out) {
    double zend = zend_start, zz = zend_start;
    for (int i = 0; i < n; ++i) {
        zz = zend;
        zend = zr * zz;
        const double dz = 0.25 * (zend - zz);
        zz += dz;
        zz += dz;
        zz += dz;
        zz += dz;
    }
    *z_last = zz;
    *zend_out = zend;
}

BQP_HD double cheb_eval(const double* c, int terms, double lo, double hi, double t) {
    const double x = (2.0 * t - (hi + lo)) / (hi - lo);
    double b1 = 0.0, b2 = 0.0;
    for (int j = terms - 1; j >= 1; --j) {
        const double tmp = fma(2.0 * x, b1, -b2) + c[j];
        b2 = b1;
        b1 = tmp;
    }
    return fma(x, b1, -b2) + c[0];
}

BQP_HD bool fit_covers(const JbFit* f, double tinf) {
    return f != nullptr && f->valid && tinf >= f->lo && tinf <= f->hi;
}

BQP_HD double mbar(double z) {
    double dz = z - 100.0;
    return dz * (dz * (dz * (dz * (dz * (dz * JBT(kCxamb)[6] + JBT(kCxamb)[5]) + JBT(kCxamb)[4]) + JBT(kCxamb)[3]) +
                       JBT(kCxamb)[2]) + JBT(kCxamb)[1]) + JBT(kCxamb)[0];
}
BQP_HD double grav(double z) {
    double s = 1.0 + z / kEarthR;
    return kG0 / (s * s);
}
BQP_HD double five_halves(double x) { return x * x * sqrt(x); }

// Local temperature profile: below the 125 km break a polynomial in dz, above
// it the arctangent approach to the exospheric temperature.
BQP_HD double local_temp(double z, const double* tc) {
    double dz = z - 125.0;
    if (dz <= 0.0) return ((-9.8204695e-6 * dz - 7.3039742e-4) * dz * dz + 1.0) * dz * tc[1] + tc[0];
    return tc[0] + tc[2] * atan(tc[3] * dz * (1.0 + 4.5e-6 * five_halves(dz)));
}

// Temperature correction for local solar time and latitude (the DTC term).
BQP_HD double dtc_correction(double f10, double st_hour, double cs, double alt) {
    if (!(alt >= 120.0 && alt <= 800.0)) return 0.0;
    double st = st_hour / 24.0;
    double fs = (f10 - 100.0) / 100.0;
    const double* c = JBT(kCdt);
    const double* b = JBT(kBdt);
    double p1c = c[0] + fs * (c[1] + st * (c[2] + st * (c[3] + st * (c[4] + st * (c[5] + st * c[6]))))) +
                 cs * st * (c[7] + st * (c[8] + st * (c[9] + st * (c[10] + st * c[11])))) +
                 cs * (c[12] + fs * (c[13] + st * (c[14] + st * c[15])));
    double p2c = c[16] + st * cs * (c[17] + st * (c[18] + st * c[19])) +
                 fs * cs * (c[20] + st * (c[21] + st * c[22]));
    double p2b = b[12] + st * (b[13] + st * (b[14] + st * (b[15] + st * (b[16] + st * b[17]))));
    double p1b_base = b[0] + fs * (b[1] + st * (b[2] + st * (b[3] + st * (b[4] + st * (b[5] + st * b[6])))));
    double p1b_st = st * (b[7] + st * (b[8] + st * (b[9] + st * (b[10] + st * b[11]))));
    if (alt > 600.0) {
        double aa = p1b_base + cs * (p1b_st + 6.0 * p2b + b[18]);
        double bb = cs * p2b;
        double cc = -(3.0 * aa + 4.0 * bb) / 4.0;
        double dd = (aa + bb) / 4.0;
        double zp = (alt - 600.0) / 100.0;
        return aa + zp * (bb + zp * (cc + zp * dd));
    } else if (alt > 300.0) {
        return p1b_base + cs * (p1b_st + alt * p2b / 100.0 + b[18]);
    } else if (alt > 240.0) {
        double bb = p1c;
        double aa = 0.8 * bb + p2c;
        double d300 = p1b_base + cs * (p1b_st + 3.0 * p2b + b[18]);
        double d300dz = cs * p2b;
        double cc = 3.0 * d300 - d300dz - 3.0 * aa - 2.0 * bb;
        double dd = d300 - aa - bb - cc;
        double zp = (alt - 240.0) / 60.0;
        return aa + zp * (bb + zp * (cc + zp * dd));
    } else if (alt > 200.0) {
        return p1c * (alt - 200.0) / 50.0 + p2c;
    } else {
        double cc = 3.0 * p2c - p1c;
        double dd = p2c - cc;
        double zp = (alt - 120.0) / 80.0;
        return zp * zp * (cc + dd * zp);
    }
}

// Day of year from a UTC MJD, the model's own 4-year-cycle arithmetic.
BQP_HD double day_of_year(double mjd, bool* ok) {
    double d1950 = mjd - 33281.0;
    double tr = trunc(d1950);
    if (!(fabs(tr) < 2.0e9)) {
        *ok = false;
        return 0.0;
    }
    long long iy = (long long)tr;
    double frac = d1950 - (double)iy;
    iy += 364;
    long long it = iy / 1461;
    iy -= it * 1461;
    it = iy / 365;
    if (it > 3) it = 3;
    iy = iy - 365 * it + 1;
    *ok = true;
    return (double)iy + frac;
}

// One Boole-rule sweep of `n` log-spaced intervals from z (exclusive carry
// `ain` at the start node).  kind 0: integrand mbar*g/T, else g/T.
struct Sweep {
    double sum, z, zend, tloc, gravl, mb, ain;
};

BQP_HD Sweep boole_sweep(double z, double zend_start, double zr, int n, double ain, bool with_mbar,
                         const double* tc) {
    Sweep s;
    s.sum = 0.0;
    s.zend = zend_start;
    s.z = z;
    s.tloc = 0.0;
    s.gravl = 0.0;
    s.mb = 0.0;
    for (int i = 0; i < n; ++i) {
        double zz = s.zend;
        s.zend = zr * zz;
        double dz = 0.25 * (s.zend - zz);
        double sum1 = kW0 * ain;
#pragma unroll
        for (int j = 1; j < 5; ++j) {
            zz += dz;
            s.tloc = local_temp(zz, tc);
            s.gravl = grav(zz);
            if (with_mbar) {
                s.mb = mbar(zz);
                ain = s.mb * s.gravl / s.tloc;
            } else {
                ain = s.gravl / s.tloc;
            }
            double w = (j == 1 || j == 3) ? kW1 : (j == 2 ? kW2 : kW0);
            sum1 += w * ain;
        }
        s.sum += dz * sum1;
        s.z = zz;
    }
    s.ain = ain;
    return s;
}

// Density (kg/m^3) for: UTC MJD, solar declination, local hour angle of the
// satellite relative to the Sun (rad), geocentric latitude (rad), altitude
// (m) and the driver set.  Non-positive returns are the error codes above.
BQP_HD double density(double mjd, double sun_dec, double hour_angle, double lat, double alt_m,
                      const Drivers& d, const JbFit* fit = nullptr) {
    if (!isfinite(mjd) || !isfinite(sun_dec) || !isfinite(hour_angle) || !isfinite(lat) ||
        !isfinite(alt_m) || !isfinite(d.f10) || !isfinite(d.f10b) || !isfinite(d.s10) ||
        !isfinite(d.s10b) || !isfinite(d.m10) || !isfinite(d.m10b) || !isfinite(d.y10) ||
        !isfinite(d.y10b) || !isfinite(d.dtc))
        return kErrNonFinite;
    if (alt_m < 90000.0) return kErrAltitude;
    if (!(sun_dec >= -kPi / 2 && sun_dec <= kPi / 2) || !(lat >= -kPi / 2 && lat <= kPi / 2))
        return kErrAngle;
    if (d.f10 <= 0.0 || d.f10b <= 0.0 || d.s10 <= 0.0 || d.s10b <= 0.0 || d.m10 <= 0.0 ||
        d.m10b <= 0.0 || d.y10 <= 0.0 || d.y10b <= 0.0)
        return kErrIndex;
    double alt = alt_m / 1000.0;
    // exospheric temperature
    double fn = fmin(pow(d.f10b / 240.0, 0.25), 1.0);
    double fsb = d.f10b * fn + d.s10b * (1.0 - fn);
    double tsubc = 392.4 + 3.227 * fsb + 0.298 * (d.f10 - d.f10b) + 2.259 * (d.s10 - d.s10b) +
                   0.312 * (d.m10 - d.m10b) + 0.178 * (d.y10 - d.y10b);
    double eta = 0.5 * fabs(lat - sun_dec);
    double theta = 0.5 * fabs(lat + sun_dec);
    double h = hour_angle;
    if (!(h >= 0.0 && h < kTwoPi)) {
        if (h < 0.0 && h > -kTwoPi) {
            h += kTwoPi;
        } else {
            h = fmod(h, kTwoPi);
            if (h < 0.0) h += kTwoPi;
        }
    }
    double tau = h - 0.64577182 + 0.10471976 * sin(h + 0.75049158);
    double st_hour = ((h + kPi) * (180.0 / kPi)) / 15.0;
    if (st_hour >= 24.0) st_hour -= 24.0;
    else if (st_hour < 0.0) st_hour += 24.0;
    double slat, clat;
    sincos(lat, &slat, &clat);
    double cos_eta = five_halves(cos(eta));
    double sin_theta = five_halves(sin(theta));
    double cos_tau = fabs(cos(0.5 * tau));
    double df = sin_theta + (cos_eta - sin_theta) * cos_tau * cos_tau * cos_tau;
    double tsubl = tsubc * (1.0 + 0.31 * df);
    double tinf = tsubl + d.dtc + dtc_correction(d.f10, st_hour, clat, alt);
    double tsubx = 444.3807 + 0.02385 * tinf - 392.8292 * exp(-0.0021357 * tinf);
    double gsubx = 0.054285714 * (tsubx - 183.0);
    double tc[4];
    tc[0] = tsubx;
    tc[1] = gsubx;
    tc[2] = (tinf - tsubx) / (kPi / 2);
    tc[3] = gsubx / tc[2];
    // 90 km -> min(alt, 105 km)
    const double z1 = 90.0;
    double al, zr;
    int n;
    const double mb1 = mbar(z1);
    const double tloc1 = local_temp(z1, tc);
    const bool use_fit = fit_covers(fit, tinf);
    Sweep lo;
    if (use_fit && alt >= 105.0) {
        lo.sum = cheb_eval(fit->low, fit->terms, fit->lo, fit->hi, tinf);
        lo.z = fit->low_z;
        lo.zend = fit->low_zend;
        lo.mb = fit->low_mb2;
        lo.gravl = fit->low_gravl;
        lo.tloc = local_temp(lo.z, tc);
    } else {
        al = log(fmin(alt, 105.0) / z1);
        n = 1 + (int)floor(al / kLnStepLower);
        zr = exp(al / n);
        lo = boole_sweep(z1, z1, zr, n, mb1 * grav(z1) / tloc1, true, tc);
    }
    double mb2 = lo.mb, tloc2 = lo.tloc;
    double rho = 3.46e-6 * mb2 * tloc1 / exp(lo.sum / kRstar) / (mb1 * tloc2);
    double anm = kAvogadro * rho;
    double an = anm / mb2;
    double fact2 = anm / 28.960;
    double fac[5] = {JBT(kFrac)[0] * fact2, fact2 * (1.0 + JBT(kFrac)[1]) - an, 2.0 * (an - fact2),
                     JBT(kFrac)[2] * fact2, JBT(kFrac)[3] * fact2};
    double aln[6];
    for (int i = 0; i < 5; ++i) aln[i] = fac[i] < 0.0 ? NAN : log(fac[i]);
    double z = lo.z;
    if (alt <= 105.0) {
        aln[5] = aln[4] - 25.0;
    } else {
        // 105 km -> min(alt, 500 km)
        Sweep mid;
        if (use_fit && alt >= 500.0) {
            mid.sum = cheb_eval(fit->mid, fit->terms, fit->lo, fit->hi, tinf);
            mid.z = fit->mid_z;
            mid.zend = fit->mid_zend;
            mid.tloc = local_temp(mid.z, tc);
            mid.gravl = fit->mid_gravl;
            mid.ain = mid.gravl / mid.tloc;
        } else {
            al = log(fmin(alt, 500.0) / z);
            n = 1 + (int)floor(al / kLnStepMiddle);
            zr = exp(al / n);
            mid = boole_sweep(z, lo.zend, zr, n, lo.gravl / tloc2, false, tc);
        }
        double tloc3 = mid.tloc;
        z = mid.z;
        // between 500 km and alt (hydrogen is anchored at 500 km)
        al = log(fmax(alt, 500.0) / z);
        n = 1 + (int)floor(al / (alt > 500.0 ? kLnStepUpper : kLnStepMiddle));
        zr = exp(al / n);
        Sweep up = boole_sweep(z, mid.zend, zr, n, mid.ain, false, tc);
        double tloc4 = up.tloc;
        z = up.z;
        double altr, hsign;
        if (alt <= 500.0) {
            altr = log(tloc3 / tloc2);
            fact2 = mid.sum / kRstar;
            hsign = 1.0;
        } else {
            altr = log(tloc4 / tloc2);
            fact2 = (mid.sum + up.sum) / kRstar;
            hsign = -1.0;
        }
        for (int i = 0; i < 4; ++i) aln[i] = aln[i] - altr - fact2 * JBT(kAmw)[i];
        aln[4] = aln[4] - (1.0 - 0.38) * altr - fact2 * JBT(kAmw)[4];
        double al10t5 = log10(tinf);
        double alnh5 = (5.5 * al10t5 - 39.40) * al10t5 + 73.13;
        aln[5] = kLn10 * (alnh5 + 6.0) + hsign * (log(tloc4 / tloc3) + up.sum * JBT(kAmw)[5] / kRstar);
    }
    // seasonal-latitudinal variation
    double years = (mjd - 36204.0) / 365.2422;
    double capphi = years - trunc(years);
    if (capphi == 0.0) capphi = copysign(0.0, years);
    double sgn = lat >= 0.0 ? 1.0 : -1.0;
    double hm90 = alt - 90.0;
    double dlrsl = 0.02 * hm90 * exp(-0.045 * hm90) * sgn * sin(kTwoPi * capphi + 1.72) * slat * slat;
    // semiannual variation
    double dlrsa = 0.0;
    if (z < 2000.0) {
        bool ok = true;
        double day = day_of_year(mjd, &ok);
        if (!ok) return kErrDomain;
        double htz = alt / 1000.0;
        double fsmb = d.f10b - 0.70 * d.s10b - 0.04 * d.m10b;
        double fzz = JBT(kFzm)[0] + JBT(kFzm)[1] * fsmb + JBT(kFzm)[2] * fsmb * htz + JBT(kFzm)[3] * fsmb * htz * htz +
                     JBT(kFzm)[4] * fsmb * fsmb * htz;
        fsmb = d.f10b - 0.75 * d.s10b - 0.37 * d.m10b;
        double s1, c1;
        sincos(kTwoPi * (day - 1.0) / 365.0, &s1, &c1);
        double s2 = 2.0 * s1 * c1, c2 = c1 * c1 - s1 * s1;
        double gtz = JBT(kGtm)[0] + JBT(kGtm)[1] * s1 + JBT(kGtm)[2] * c1 + JBT(kGtm)[3] * s2 + JBT(kGtm)[4] * c2 +
                     JBT(kGtm)[5] * fsmb + JBT(kGtm)[6] * fsmb * s1 + JBT(kGtm)[7] * fsmb * c1 + JBT(kGtm)[8] * fsmb * s2 +
                     JBT(kGtm)[9] * fsmb * c2;
        dlrsa = fmax(fzz, 1.0e-6) * gtz;
    }
    double dlr = kLn10 * (dlrsl + dlrsa);
    double sumnm = 0.0;
    for (int i = 0; i < 6; ++i) sumnm += exp(aln[i] + dlr) * JBT(kAmw)[i];
    rho = sumnm / kAvogadro;
    double fex = 1.0;
    if (alt >= 1000.0 && alt < 1500.0) {
        double zeta = (alt - 1000.0) * 0.002;
        double f15c = JBT(kCht)[0] + JBT(kCht)[1] * d.f10b + JBT(kCht)[2] * 1500.0 + JBT(kCht)[3] * d.f10b * 1500.0;
        double f15cz = (JBT(kCht)[2] + JBT(kCht)[3] * d.f10b) * 500.0;
        double fex2 = 3.0 * f15c - f15cz - 3.0;
        double fex3 = f15cz - 2.0 * f15c + 2.0;
        fex = 1.0 + zeta * zeta * (fex2 + fex3 * zeta);
    } else if (alt >= 1500.0) {
        fex = JBT(kCht)[0] + JBT(kCht)[1] * d.f10b + JBT(kCht)[2] * alt + JBT(kCht)[3] * d.f10b * alt;
    }
    double out = rho * fex;
    if (!(isfinite(out) && out > 0.0)) return kErrDomain;
    return out;
}

// ------------------------------------------------------------------------
// The reference's coarse quadrature profiles, atm_model 5, 6 and 7
// (jb_rs/src/jb2008.rs:365-460, 770-838; jb_density 2353-2624): fewer, wider
// Boole panels, the five species carried as factor x exp(log offset)
// (jb2008.rs:2420-2455) and a compensated species sum (2584-2607).  Model 7
// (the reference's default) also takes the one-panel upper segment's step
// ratio directly (2049-2058), drops the seasonal-latitudinal term at and
// above 800 km (2372-2381) and replaces the two fixed plans (90-105 km,
// 105-500 km) by degree-14 series in the exospheric temperature inside
// [500, 2600] K (497-838).  Its costly part is small: above 500 km five
// series, one upper panel (four arctangents) and the species; below, six
// 105-500 km panels at most.
constexpr double kV7TexoLo = 500.0, kV7TexoHi = 2600.0;
// jb2008.rs:645-762 (the reference's fits of its fixed-plan walkers), lowest
// coefficient first
BQP_JB_TABLE(kV7Sub2Lower, 15, {2.08308130371611e1, -2.2813199227110412e-1, 1.4879239222099155e-1,
                                -1.139133002344331e-1, 6.719889370881822e-2, -3.2986547523035745e-2,
                                1.4447262123974028e-2, -5.996731588024651e-3, 2.506977417579703e-3,
                                -1.1683682791648784e-3, 5.31782582941462e-4, -1.236948769467779e-4,
                                4.605879140433796e-5, -1.0052021764385242e-4, 4.8436805479216456e-5})
BQP_JB_TABLE(kV7Tloc2, 15, {2.2451892791577825e2, 8.361916544062648e0, -5.270934320812583e0, 3.939997041634312e0,
                            -2.208846067908349e0, 9.906609315622759e-1, -3.7025703779179586e-1,
                            1.186132114284294e-1, -3.324856853041033e-2, 8.285607849008118e-3,
                            -1.857998341613101e-3, 3.7710530702575305e-4, -7.049765582078043e-5,
                            1.331415410018169e-5, -2.125129463136452e-6})
BQP_JB_TABLE(kV7Sub2Middle, 15, {3.2040046352489187e0, -1.379154303257483e0, 9.72715573920378e-1,
                                 -6.869617534038228e-1, 4.6837996271501126e-1, -3.319992425165518e-1,
                                 2.3364063163661636e-1, -7.314250955188073e-2, 1.7496078898220538e-2,
                                 -2.2706819285120894e-1, 2.0222194979627475e-1, 1.5675573900373196e-1,
                                 -1.4292464982323266e-1, -1.0640427393729598e-1, 8.289447705809763e-2})
BQP_JB_TABLE(kV7AinMiddle, 15, {5.459640467018433e-3, -3.677621602992105e-3, 2.492908325931464e-3,
                                -1.6862184086503845e-3, 1.13828516769243e-3, -8.142832736202574e-4,
                                5.787786476720627e-4, -1.761805263267051e-4, 3.7786418569522054e-5,
                                -5.77028261806222e-4, 5.158819094236952e-4, 4.0211633550021317e-4,
                                -3.670455396068389e-4, -2.714264714701178e-4, 2.1193481991044327e-4})
BQP_JB_TABLE(kV7Tloc3, 15, {1.5437971407829077e3, 1.039876918772851e3, -4.373905347259339e0,
                            1.1486679813161453e-1, 1.5536392865018533e-1, -6.297264812830576e-2,
                            7.581060757845705e-3, 3.246438671753597e-3, -1.4342975630790944e-3,
                            -5.114031895849491e-5, 2.0780285514906778e-4, -6.117111036343099e-5,
                            -4.124441270261577e-6, 6.126914161375104e-6, -8.797891983987146e-7})

// The coarse profiles are written once for the arithmetic type R: FP64 (the
// reference's) or FP32 (the split form's density, drag_fp32).  These pick the
// math function of each type; for double they are the calls the FP64 code
// has always made.
namespace rm {
BQP_HD double log(double x) { return ::log(x); }
BQP_HD float log(float x) { return ::logf(x); }
BQP_HD double log10(double x) { return ::log10(x); }
BQP_HD float log10(float x) { return ::log10f(x); }
BQP_HD double exp(double x) { return ::exp(x); }
BQP_HD float exp(float x) { return ::expf(x); }
BQP_HD double atan(double x) { return ::atan(x); }
BQP_HD float atan(float x) { return ::atanf(x); }
BQP_HD double pow(double x, double y) { return ::pow(x, y); }
BQP_HD float pow(float x, float y) { return ::powf(x, y); }
BQP_HD double sin(double x) { return ::sin(x); }
BQP_HD float sin(float x) { return ::sinf(x); }
BQP_HD double cos(double x) { return ::cos(x); }
BQP_HD float cos(float x) { return ::cosf(x); }
BQP_HD void sincos(double x, double* s, double* c) { ::sincos(x, s, c); }
BQP_HD void sincos(float x, float* s, float* c) { ::sincosf(x, s, c); }
BQP_HD double sqrt(double x) { return ::sqrt(x); }
BQP_HD float sqrt(float x) { return ::sqrtf(x); }
BQP_HD double fma(double a, double b, double c) { return ::fma(a, b, c); }
BQP_HD float fma(float a, float b, float c) { return ::fmaf(a, b, c); }
BQP_HD double fmin(double a, double b) { return ::fmin(a, b); }
BQP_HD float fmin(float a, float b) { return ::fminf(a, b); }
BQP_HD double fmax(double a, double b) { return ::fmax(a, b); }
BQP_HD float fmax(float a, float b) { return ::fmaxf(a, b); }
BQP_HD double fabs(double x) { return ::fabs(x); }
BQP_HD float fabs(float x) { return ::fabsf(x); }
BQP_HD double floor(double x) { return ::floor(x); }
BQP_HD float floor(float x) { return ::floorf(x); }
BQP_HD double fmod(double a, double b) { return ::fmod(a, b); }
BQP_HD float fmod(float a, float b) { return ::fmodf(a, b); }
}  // namespace rm

// Estrin evaluation of a 15-term series (the reference's tree,
// jb2008.rs:561-643): pairs fused through u, u^2, u^4, u^8, the last
// coefficient joining at the u^2 level.
template <class R>
BQP_HD R v7_series(const double* cd, R u) {
    R c[15];
#pragma unroll
    for (int i = 0; i < 15; ++i) c[i] = (R)cd[i];
    const R u2 = u * u, u4 = u2 * u2, u8 = u4 * u4;
    const R a0 = rm::fma(c[1], u, c[0]), a1 = rm::fma(c[3], u, c[2]), a2 = rm::fma(c[5], u, c[4]);
    const R a3 = rm::fma(c[7], u, c[6]), a4 = rm::fma(c[9], u, c[8]), a5 = rm::fma(c[11], u, c[10]);
    const R a6 = rm::fma(c[13], u, c[12]);
    const R b0 = rm::fma(a1, u2, a0), b1 = rm::fma(a3, u2, a2), b2 = rm::fma(a5, u2, a4),
            b3 = rm::fma(c[14], u2, a6);
    return rm::fma(rm::fma(b3, u4, b2), u8, rm::fma(b1, u4, b0));
}

// Panel count of a log ratio (jb2008.rs:1515-1526); 0 on a domain error.
template <class R>
BQP_HD int coarse_panels(R log_ratio) {
    if (!(isfinite(log_ratio) && log_ratio >= (R)0) || rm::floor(log_ratio) >= (R)2147483520.0) return 0;
    return (int)rm::floor(log_ratio) + 1;
}

// mbar, grav, local_temp, dtc_correction and boole_sweep in R (the same
// expressions as the FP64 functions above)
template <class R>
BQP_HD R mbar_r(R z) {
    const double* c = JBT(kCxamb);
    const R dz = z - (R)100.0;
    return dz * (dz * (dz * (dz * (dz * (dz * (R)c[6] + (R)c[5]) + (R)c[4]) + (R)c[3]) + (R)c[2]) + (R)c[1]) +
           (R)c[0];
}
template <class R>
BQP_HD R grav_r(R z) {
    const R s = (R)1.0 + z / (R)kEarthR;
    return (R)kG0 / (s * s);
}
template <class R>
BQP_HD R local_temp_r(R z, const R* tc) {
    const R dz = z - (R)125.0;
    if (dz <= (R)0.0) return (((R)-9.8204695e-6 * dz - (R)7.3039742e-4) * dz * dz + (R)1.0) * dz * tc[1] + tc[0];
    return tc[0] + tc[2] * rm::atan(tc[3] * dz * ((R)1.0 + (R)4.5e-6 * (dz * dz * rm::sqrt(dz))));
}
template <class R>
BQP_HD R dtc_correction_r(R f10, R st_hour, R cs, R alt) {
    if (!(alt >= (R)120.0 && alt <= (R)800.0)) return (R)0.0;
    const R st = st_hour / (R)24.0;
    const R fs = (f10 - (R)100.0) / (R)100.0;
    R c[23], b[19];
#pragma unroll
    for (int i = 0; i < 23; ++i) c[i] = (R)JBT(kCdt)[i];
#pragma unroll
    for (int i = 0; i < 19; ++i) b[i] = (R)JBT(kBdt)[i];
    const R p1c = c[0] + fs * (c[1] + st * (c[2] + st * (c[3] + st * (c[4] + st * (c[5] + st * c[6]))))) +
                  cs * st * (c[7] + st * (c[8] + st * (c[9] + st * (c[10] + st * c[11])))) +
                  cs * (c[12] + fs * (c[13] + st * (c[14] + st * c[15])));
    const R p2c = c[16] + st * cs * (c[17] + st * (c[18] + st * c[19])) +
                  fs * cs * (c[20] + st * (c[21] + st * c[22]));
    const R p2b = b[12] + st * (b[13] + st * (b[14] + st * (b[15] + st * (b[16] + st * b[17]))));
    const R p1b_base = b[0] + fs * (b[1] + st * (b[2] + st * (b[3] + st * (b[4] + st * (b[5] + st * b[6])))));
    const R p1b_st = st * (b[7] + st * (b[8] + st * (b[9] + st * (b[10] + st * b[11]))));
    if (alt > (R)600.0) {
        const R aa = p1b_base + cs * (p1b_st + (R)6.0 * p2b + b[18]);
        const R bb = cs * p2b;
        const R cc = -((R)3.0 * aa + (R)4.0 * bb) / (R)4.0;
        const R dd = (aa + bb) / (R)4.0;
        const R zp = (alt - (R)600.0) / (R)100.0;
        return aa + zp * (bb + zp * (cc + zp * dd));
    } else if (alt > (R)300.0) {
        return p1b_base + cs * (p1b_st + alt * p2b / (R)100.0 + b[18]);
    } else if (alt > (R)240.0) {
        const R bb = p1c;
        const R aa = (R)0.8 * bb + p2c;
        const R d300 = p1b_base + cs * (p1b_st + (R)3.0 * p2b + b[18]);
        const R d300dz = cs * p2b;
        const R cc = (R)3.0 * d300 - d300dz - (R)3.0 * aa - (R)2.0 * bb;
        const R dd = d300 - aa - bb - cc;
        const R zp = (alt - (R)240.0) / (R)60.0;
        return aa + zp * (bb + zp * (cc + zp * dd));
    } else if (alt > (R)200.0) {
        return p1c * (alt - (R)200.0) / (R)50.0 + p2c;
    } else {
        const R cc = (R)3.0 * p2c - p1c;
        const R dd = p2c - cc;
        const R zp = (alt - (R)120.0) / (R)80.0;
        return zp * zp * (cc + dd * zp);
    }
}
template <class R>
struct SweepR {
    R sum, z, zend, tloc, gravl, mb, ain;
};
template <class R>
BQP_HD SweepR<R> boole_sweep_r(R z, R zend_start, R zr, int n, R ain, bool with_mbar, const R* tc) {
    SweepR<R> s;
    s.sum = (R)0.0;
    s.zend = zend_start;
    s.z = z;
    s.tloc = (R)0.0;
    s.gravl = (R)0.0;
    s.mb = (R)0.0;
    for (int i = 0; i < n; ++i) {
        R zz = s.zend;
        s.zend = zr * zz;
        const R dz = (R)0.25 * (s.zend - zz);
        R sum1 = (R)kW0 * ain;
#pragma unroll
        for (int j = 1; j < 5; ++j) {
            zz += dz;
            s.tloc = local_temp_r(zz, tc);
            s.gravl = grav_r(zz);
            if (with_mbar) {
                s.mb = mbar_r(zz);
                ain = s.mb * s.gravl / s.tloc;
            } else {
                ain = s.gravl / s.tloc;
            }
            const R w = (j == 1 || j == 3) ? (R)kW1 : (j == 2 ? (R)kW2 : (R)kW0);
            sum1 += w * ain;
        }
        s.sum += dz * sum1;
        s.z = zz;
    }
    s.ain = ain;
    return s;
}

// As density(), for atm_model 5, 6 or 7, in R after the input checks.  FP64:
// the reference's arithmetic.  FP32: the split form's density; its relative
// error (~1e-6: the exponents reach ~45) moves the drag acceleration by
// ~1e-15 km/s^2, and number densities (~1e21 per m^3 at 90 km) stay well
// inside FP32's range.  The epoch terms (fractional year, day of year) are
// kept in FP64, since an MJD does not fit FP32.
template <class R>
BQP_HD double density_coarse_r(double mjd, double sun_dec, double hour_angle, double lat_in, double alt_m,
                               const Drivers& din, int model) {
    const R step_lower = (R)0.040, step_middle = model == 5 ? (R)0.100 : (R)0.300;
    const R step_upper = model == 5 ? (R)0.300 : (R)0.700;
    const bool v7 = model == 7;
    if (!isfinite(mjd) || !isfinite(sun_dec) || !isfinite(hour_angle) || !isfinite(lat_in) ||
        !isfinite(alt_m) || !isfinite(din.f10) || !isfinite(din.f10b) || !isfinite(din.s10) ||
        !isfinite(din.s10b) || !isfinite(din.m10) || !isfinite(din.m10b) || !isfinite(din.y10) ||
        !isfinite(din.y10b) || !isfinite(din.dtc))
        return kErrNonFinite;
    if (alt_m < 90000.0) return kErrAltitude;
    if (!(sun_dec >= -kPi / 2 && sun_dec <= kPi / 2) || !(lat_in >= -kPi / 2 && lat_in <= kPi / 2))
        return kErrAngle;
    if (din.f10 <= 0.0 || din.f10b <= 0.0 || din.s10 <= 0.0 || din.s10b <= 0.0 || din.m10 <= 0.0 ||
        din.m10b <= 0.0 || din.y10 <= 0.0 || din.y10b <= 0.0)
        return kErrIndex;
    const R alt = (R)(alt_m / 1000.0);
    const R lat = (R)lat_in, sdec = (R)sun_dec;
    const R f10 = (R)din.f10, f10b = (R)din.f10b, s10 = (R)din.s10, s10b = (R)din.s10b, m10 = (R)din.m10,
            m10b = (R)din.m10b, y10 = (R)din.y10, y10b = (R)din.y10b, dtc_k = (R)din.dtc;
    const R pi = (R)kPi, two_pi = (R)kTwoPi;
    // exospheric temperature and profile, as density()
    const R fn = rm::fmin(rm::pow(f10b / (R)240.0, (R)0.25), (R)1.0);
    const R fsb = f10b * fn + s10b * ((R)1.0 - fn);
    const R tsubc = (R)392.4 + (R)3.227 * fsb + (R)0.298 * (f10 - f10b) + (R)2.259 * (s10 - s10b) +
                    (R)0.312 * (m10 - m10b) + (R)0.178 * (y10 - y10b);
    const R eta = (R)0.5 * rm::fabs(lat - sdec);
    const R theta = (R)0.5 * rm::fabs(lat + sdec);
    R h = (R)hour_angle;
    if (!(h >= (R)0.0 && h < two_pi)) {
        if (h < (R)0.0 && h > -two_pi) {
            h += two_pi;
        } else {
            h = rm::fmod(h, two_pi);
            if (h < (R)0.0) h += two_pi;
        }
    }
    const R tau = h - (R)0.64577182 + (R)0.10471976 * rm::sin(h + (R)0.75049158);
    R st_hour = ((h + pi) * ((R)180.0 / pi)) / (R)15.0;
    if (st_hour >= (R)24.0) st_hour -= (R)24.0;
    else if (st_hour < (R)0.0) st_hour += (R)24.0;
    R slat, clat;
    rm::sincos(lat, &slat, &clat);
    const R ce = rm::cos(eta), sn = rm::sin(theta);
    const R cos_eta = ce * ce * rm::sqrt(ce);
    const R sin_theta = sn * sn * rm::sqrt(sn);
    const R cos_tau = rm::fabs(rm::cos((R)0.5 * tau));
    const R df = sin_theta + (cos_eta - sin_theta) * cos_tau * cos_tau * cos_tau;
    const R tsubl = tsubc * ((R)1.0 + (R)0.31 * df);
    const R tinf = tsubl + dtc_k + dtc_correction_r(f10, st_hour, clat, alt);
    const R tsubx = (R)444.3807 + (R)0.02385 * tinf - (R)392.8292 * rm::exp((R)-0.0021357 * tinf);
    const R gsubx = (R)0.054285714 * (tsubx - (R)183.0);
    R tc[4];
    tc[0] = tsubx;
    tc[1] = gsubx;
    tc[2] = (tinf - tsubx) / (pi / (R)2);
    tc[3] = gsubx / tc[2];
    // the fit domain is judged on Texo rebuilt from the profile (jb2008.rs:521-524)
    const R texo = tc[0] + tc[2] * (pi / (R)2);
    const bool fit_in = v7 && texo >= (R)kV7TexoLo && texo <= (R)kV7TexoHi;
    const R u = (R)2.0 * (texo - (R)kV7TexoLo) / (R)(kV7TexoHi - kV7TexoLo) - (R)1.0;

    // 90 km -> min(alt, 105 km): four panels at and above 105 km (the fixed plan)
    const R z1 = (R)90.0;
    const R mb1 = mbar_r(z1);
    const R tloc1 = local_temp_r(z1, tc);
    const bool lower_planned = alt >= (R)105.0;
    R al = rm::log(rm::fmin(alt, (R)105.0) / z1);
    int n = coarse_panels(al / step_lower);
    if (n == 0) return kErrDomain;
    SweepR<R> lo = boole_sweep_r(z1, z1, rm::exp(al / (R)n), n, mb1 * grav_r(z1) / tloc1, true, tc);
    if (fit_in && lower_planned) {
        lo.sum = v7_series(JBT(kV7Sub2Lower), u);
        lo.tloc = v7_series(JBT(kV7Tloc2), u);
    }
    const R mb2 = lo.mb, tloc2 = lo.tloc;
    const R rstar = (R)kRstar, avog = (R)kAvogadro;
    R rho = (R)3.46e-6 * mb2 * tloc1 / rm::exp(lo.sum / rstar) / (mb1 * tloc2);
    const R anm = avog * rho;
    const R an = anm / mb2;
    R fact2 = anm / (R)28.960;
    R factor[6] = {(R)JBT(kFrac)[0] * fact2, fact2 * ((R)1.0 + (R)JBT(kFrac)[1]) - an, (R)2.0 * (an - fact2),
                   (R)JBT(kFrac)[2] * fact2, (R)JBT(kFrac)[3] * fact2, (R)1.0};
#pragma unroll
    for (int i = 0; i < 6; ++i)
        if (factor[i] < (R)0.0) factor[i] = (R)NAN;  // jb2008.rs:2304-2310
    R offset[6] = {(R)0.0, (R)0.0, (R)0.0, (R)0.0, (R)0.0, (R)0.0};
    R z = lo.z;
    if (alt <= (R)105.0) {
        factor[5] = factor[4];
        offset[5] = offset[4] - (R)25.0;
    } else {
        // 105 km -> min(alt, 500 km): the fixed six-panel plan at and above 500 km
        al = rm::log(rm::fmin(alt, (R)500.0) / z);
        n = coarse_panels(al / step_middle);
        if (n == 0) return kErrDomain;
        SweepR<R> mid = boole_sweep_r(z, lo.zend, rm::exp(al / (R)n), n, lo.gravl / tloc2, false, tc);
        if (fit_in && lower_planned && alt >= (R)500.0) {
            mid.sum = v7_series(JBT(kV7Sub2Middle), u);
            mid.ain = v7_series(JBT(kV7AinMiddle), u);
            mid.tloc = v7_series(JBT(kV7Tloc3), u);
        }
        const R tloc3 = mid.tloc;
        z = mid.z;
        // between 500 km and alt (jb2008.rs:2032-2085)
        const R ratio = rm::fmax(alt, (R)500.0) / z;
        const R alu = rm::fmax(rm::log(ratio), (R)0.0);
        n = coarse_panels(alu / (alt > (R)500.0 ? step_upper : step_middle));
        if (n == 0) return kErrDomain;
        const R zr = (v7 && n == 1) ? rm::fmax(ratio, (R)1.0) : rm::exp(alu / (R)n);
        SweepR<R> up = boole_sweep_r(z, mid.zend, zr, n, mid.ain, false, tc);
        const R tloc4 = up.tloc;
        z = up.z;
        R altr, hsign;
        if (alt <= (R)500.0) {
            fact2 = mid.sum / rstar;
            altr = rm::log(tloc3 / tloc2);
            hsign = (R)1.0;
        } else {
            fact2 = (mid.sum + up.sum) / rstar;
            altr = rm::log(tloc4 / tloc2);
            hsign = (R)-1.0;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) offset[i] = offset[i] - altr - fact2 * (R)JBT(kAmw)[i];
        offset[4] = offset[4] - ((R)1.0 - (R)0.38) * altr - fact2 * (R)JBT(kAmw)[4];
        const R al10t5 = rm::log10(tinf);
        const R alnh5 = ((R)5.5 * al10t5 - (R)39.40) * al10t5 + (R)73.13;
        offset[5] = (R)kLn10 * (alnh5 + (R)6.0) +
                    hsign * (rm::log(tloc4 / tloc3) + up.sum * (R)JBT(kAmw)[5] / rstar);
    }
    // seasonal-latitudinal term, cut at 800 km by model 7
    R dlrsl = (R)0.0;
    if (!(v7 && alt >= (R)800.0)) {
        const double years = (mjd - 36204.0) / 365.2422;
        double capphi = years - ::trunc(years);
        if (capphi == 0.0) capphi = ::copysign(0.0, years);
        const R sgn = lat_in >= 0.0 ? (R)1.0 : (R)-1.0;
        const R hm90 = alt - (R)90.0;
        dlrsl = (R)0.02 * hm90 * rm::exp((R)-0.045 * hm90) * sgn * rm::sin((R)(kTwoPi * capphi + 1.72)) * slat *
                slat;
    }
    // semiannual term (jb2008.rs:3436-3461)
    R dlrsa = (R)0.0;
    if (z < (R)2000.0) {
        bool ok = true;
        const double day = day_of_year(mjd, &ok);
        if (!ok) return kErrDomain;
        R fzm[5], gtm[10];
#pragma unroll
        for (int i = 0; i < 5; ++i) fzm[i] = (R)JBT(kFzm)[i];
#pragma unroll
        for (int i = 0; i < 10; ++i) gtm[i] = (R)JBT(kGtm)[i];
        const R htz = alt / (R)1000.0;
        const R fz = f10b - (R)0.70 * s10b - (R)0.04 * m10b;
        const R fzz = fzm[0] + fz * (fzm[1] + htz * (fzm[2] + fzm[3] * htz + fzm[4] * fz));
        const R fg = f10b - (R)0.75 * s10b - (R)0.37 * m10b;
        R s1, c1;
        rm::sincos((R)(kTwoPi * (day - 1.0) / 365.0), &s1, &c1);
        const R s2 = (R)2.0 * s1 * c1, c2 = c1 * c1 - s1 * s1;
        const R gtz = gtm[0] + gtm[1] * s1 + gtm[2] * c1 + gtm[3] * s2 + gtm[4] * c2 +
                      fg * (gtm[5] + gtm[6] * s1 + gtm[7] * c1 + gtm[8] * s2 + gtm[9] * c2);
        dlrsa = rm::fmax(fzz, (R)1.0e-6) * gtz;
    }
    const R dlr = (R)kLn10 * (dlrsl + dlrsa);
    // compensated species sum
    R sum = (R)0.0, comp = (R)0.0, simple = (R)0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const R term = factor[i] * rm::exp(offset[i] + dlr) * (R)JBT(kAmw)[i];
        const R tmp = term - comp;
        const R next = sum + tmp;
        comp = (next - sum) - tmp;
        sum = next;
        simple += term;
    }
    R fs = sum - comp;
    if (isnan(fs) && isinf(simple)) fs = simple;
    rho = fs / avog;
    R fex = (R)1.0;
    if (alt >= (R)1000.0 && alt < (R)1500.0) {
        R cht[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) cht[i] = (R)JBT(kCht)[i];
        const R zeta = (alt - (R)1000.0) * (R)0.002;
        const R f15c = cht[0] + cht[1] * f10b + cht[2] * (R)1500.0 + cht[3] * f10b * (R)1500.0;
        const R f15cz = (cht[2] + cht[3] * f10b) * (R)500.0;
        const R fex2 = (R)3.0 * f15c - f15cz - (R)3.0;
        const R fex3 = f15cz - (R)2.0 * f15c + (R)2.0;
        fex = (R)1.0 + zeta * zeta * (fex2 + fex3 * zeta);
    } else if (alt >= (R)1500.0) {
        fex = (R)JBT(kCht)[0] + (R)JBT(kCht)[1] * f10b + (R)JBT(kCht)[2] * alt + (R)JBT(kCht)[3] * f10b * alt;
    }
    const double out = (double)(rho * fex);
    if (!(isfinite(out) && out > 0.0)) return kErrDomain;
    return out;
}

BQP_HD double density_coarse(double mjd, double sun_dec, double hour_angle, double lat, double alt_m,
                             const Drivers& d, int model) {
    return density_coarse_r<double>(mjd, sun_dec, hour_angle, lat, alt_m, d, model);
}

// The density of atm_model 4 (exact, with the optional sweep fits) or 5-7.
BQP_HD double density_model(double mjd, double sun_dec, double hour_angle, double lat, double alt_m,
                            const Drivers& d, int model, const JbFit* fit = nullptr) {
    if (model == 4) return density(mjd, sun_dec, hour_angle, lat, alt_m, d, fit);
    return density_coarse(mjd, sun_dec, hour_angle, lat, alt_m, d, model);
}

#ifdef __CUDACC__
// ------------------------------------------------------------------------
// Lane-group form for the drag kernel: the density of one state is computed
// by a group of L consecutive lanes.  Every lane walks the same log-spaced
// interval chain (bit-identical node positions); lane q evaluates the Boole
// nodes of intervals i = q (mod L), including the node carried in from
// interval i-1, recomputed -- the same function at the same altitude, so the
// same value.  Partial sums meet in a group-masked shuffle.  All lanes of a
// group hold the same inputs, so they branch together.
typedef Sweep SweepG;

BQP_HD double node_ain(double z, const double* tc, bool with_mbar, double* tloc, double* gravl, double* mb) {
    *tloc = local_temp(z, tc);
    *gravl = grav(z);
    if (with_mbar) {
        *mb = mbar(z);
        return *mb * *gravl / *tloc;
    }
    return *gravl / *tloc;
}

template <int L>
// How the drag kernel's sweep helpers are compiled: inlined at each of their
// call sites (the default) or as one out-of-line copy each, which shrinks
// the kernel's code when instruction fetch limits it.
#ifndef BQP_JB_SWEEP_INLINE
#define BQP_JB_SWEEP_INLINE __forceinline__
#endif
__device__ BQP_JB_SWEEP_INLINE SweepG boole_sweep_group(double zend_start, double zr, int n, double ain0,
                                                    bool with_mbar, const double* tc, int q, unsigned gmask) {
    SweepG s;
    double part = 0.0;
    double zend = zend_start, zlast = zend_start;  // zlast: last node of the previous interval
    double tl = 0.0, gl = 0.0, mb = 0.0, ain_last = ain0;
    const int rounds = (n + L - 1) / L;
    for (int r = 0; r < rounds; ++r) {
        // advance the interval chain by L intervals (cheap, identical on
        // every lane) and keep this lane's interval r*L + q
        double my_start = 0.0, my_dz = 0.0, my_prev = zlast;
#pragma unroll
        for (int k = 0; k < L; ++k) {
            const int i = r * L + k;
            if (i < n) {
                double zz = zend;
                zend = zr * zz;
                const double dz = 0.25 * (zend - zz);
                if (k == q) {
                    my_start = zz;
                    my_dz = dz;
                    my_prev = zlast;
                }
                zz += dz;
                zz += dz;
                zz += dz;
                zz += dz;
                zlast = zz;
            }
        }
        // every lane evaluates its own interval's nodes together
        const int mi = r * L + q;
        if (mi < n) {
            double t_, g_, m_;
            const double carry = mi == 0 ? ain0 : node_ain(my_prev, tc, with_mbar, &t_, &g_, &m_);
            double sum1 = kW0 * carry;
            double zz = my_start;
#pragma unroll
            for (int j = 1; j < 5; ++j) {
                zz += my_dz;
                const double a = node_ain(zz, tc, with_mbar, &tl, &gl, &mb);
                sum1 += (j == 1 || j == 3 ? kW1 : (j == 2 ? kW2 : kW0)) * a;
                ain_last = a;
            }
            part += my_dz * sum1;
        }
    }
    // group reduction and the last interval's node values from its owner
#pragma unroll
    for (int off = L / 2; off > 0; off >>= 1) part += __shfl_xor_sync(gmask, part, off, L);
    const int owner = n > 0 ? (n - 1) % L : 0;
    s.sum = part;
    s.z = zlast;
    s.zend = zend;
    s.tloc = __shfl_sync(gmask, tl, owner, L);
    s.gravl = __shfl_sync(gmask, gl, owner, L);
    s.mb = __shfl_sync(gmask, mb, owner, L);
    s.ain = __shfl_sync(gmask, ain_last, owner, L);
    return s;
}

// density() evaluated by a group of L lanes (q = lane within the group,
// gmask = the group's lanes).  Same inputs, same error codes.
// A sweep of n intervals from zend_start whose sum comes from the 2-D fit c
// at (xa, xt), plus the intervals ex[0]..ex[1] walked exactly (carry ain0
// into interval 0).  The group of L lanes shares the work: lane q evaluates
// the series rows ka = q, q + L, ... in T_inf and the exact intervals
// i = q (mod L); shuffles combine them, and every lane runs the short
// series in the altitude variable and recomputes the final node.
template <int L>
__device__ BQP_JB_SWEEP_INLINE SweepG fitted_sweep(const double* c, const int32_t* ex, double xa, double xt,
                                               double zend_start, double zr, int n, double ain0, const double* tc,
                                               int q, unsigned gmask) {
    static_assert(kFit2A % L == 0, "series rows must split evenly over the lanes");
    constexpr int R = L == 1 ? 1 : kFit2A / L;
    SweepG s;
    // rows of the series in T_inf, this lane's share (one lane: each row is
    // summed where the series in altitude takes it)
    double v[R];
#pragma unroll
    for (int r = 0; r < (L == 1 ? 0 : R); ++r) {
        const double* row = c + (r * L + q) * kFit2T;
        double b1 = 0.0, b2 = 0.0;
        for (int j = kFit2T - 1; j >= 1; --j) {
            const double tmp = fma(2.0 * xt, b1, -b2) + row[j];
            b2 = b1;
            b1 = tmp;
        }
        v[r] = fma(xt, b1, -b2) + row[0];
    }
    // the node chain (every lane), this lane's exact intervals
    double zend = zend_start, zz = zend_start, zlast = zend_start, exact = 0.0;
    for (int i = 0; i < n; ++i) {
        zz = zend;
        zend = zr * zz;
        const double dz = 0.25 * (zend - zz);
        if (i >= ex[0] && i <= ex[1] && (i - ex[0]) % L == q) {
            double t_, g_, m_;
            const double carry = i == 0 ? ain0 : node_ain(zlast, tc, false, &t_, &g_, &m_);
            double sum1 = kW0 * carry, z2 = zz;
#pragma unroll
            for (int j = 1; j < 5; ++j) {
                z2 += dz;
                sum1 += (j == 1 || j == 3 ? kW1 : (j == 2 ? kW2 : kW0)) * node_ain(z2, tc, false, &t_, &g_, &m_);
            }
            exact += dz * sum1;
        }
        zz += dz;
        zz += dz;
        zz += dz;
        zz += dz;
        zlast = zz;
    }
#pragma unroll
    for (int off = L / 2; off > 0; off >>= 1) exact += __shfl_xor_sync(gmask, exact, off, L);
    // the series in the altitude variable over the gathered rows
    double a1 = 0.0, a2 = 0.0, sum = 0.0;
#pragma unroll
    for (int ka = kFit2A - 1; ka >= 0; --ka) {
        double vk;
        if constexpr (L == 1) {
            const double* row = c + ka * kFit2T;
            double b1 = 0.0, b2 = 0.0;
            for (int j = kFit2T - 1; j >= 1; --j) {
                const double tmp = fma(2.0 * xt, b1, -b2) + row[j];
                b2 = b1;
                b1 = tmp;
            }
            vk = fma(xt, b1, -b2) + row[0];
        } else {
            vk = __shfl_sync(gmask, v[ka / L], ka % L, L);
        }
        if (ka == 0) {
            sum = fma(xa, a1, -a2) + vk;
        } else {
            const double tmp = fma(2.0 * xa, a1, -a2) + vk;
            a2 = a1;
            a1 = tmp;
        }
    }
    s.z = zz;
    s.zend = zend;
    s.sum = sum + exact;
    s.tloc = local_temp(s.z, tc);
    s.gravl = grav(s.z);
    s.mb = 0.0;
    s.ain = s.gravl / s.tloc;
    return s;
}

// The fixed-node sweep fits are one table for every context (the sums depend
// only on T_inf; the node altitudes are fixed), so the density kernel of the
// stage-synchronous engine reads them from constant memory: this
// translation unit's copy, which the engine fills on the caller's stream
// before each propagation's kernels.
static __constant__ JbFit c_fixed_fit;

// The two fixed-node sums at one T_inf (cheb_eval of both series, the same
// operations): the two recurrences run in one loop as independent chains,
// unrolled so that every coefficient is a constant-bank operand.
__device__ __forceinline__ void cheb_eval_pair(double t, double* low, double* mid) {
    const JbFit& f = c_fixed_fit;
    const double x = (2.0 * t - (f.hi + f.lo)) / (f.hi - f.lo);
    double a1 = 0.0, a2 = 0.0, b1 = 0.0, b2 = 0.0;
#pragma unroll
    for (int j = kFitTerms - 1; j >= 1; --j) {
        const double ta = fma(2.0 * x, a1, -a2) + f.low[j];
        const double tb = fma(2.0 * x, b1, -b2) + f.mid[j];
        a2 = a1;
        a1 = ta;
        b2 = b1;
        b1 = tb;
    }
    *low = fma(x, a1, -a2) + f.low[0];
    *mid = fma(x, b1, -b2) + f.mid[0];
}

// fixed_fit: use the fixed-node sweep fits (c_fixed_fit) where they apply.
template <int L>
__device__ double density_group(double mjd, double sun_dec, double hour_angle, double lat, double alt_m,
                                const Drivers& d, int q, unsigned gmask, bool fixed_fit,
                                const JbFit2* fit2 = nullptr) {
    const JbFit* fit = fixed_fit ? &c_fixed_fit : nullptr;
    double code = 0.0;
    if (!isfinite(mjd) || !isfinite(sun_dec) || !isfinite(hour_angle) || !isfinite(lat) || !isfinite(alt_m) ||
        !isfinite(d.f10) || !isfinite(d.f10b) || !isfinite(d.s10) || !isfinite(d.s10b) || !isfinite(d.m10) ||
        !isfinite(d.m10b) || !isfinite(d.y10) || !isfinite(d.y10b) || !isfinite(d.dtc))
        code = kErrNonFinite;
    else if (alt_m < 90000.0)
        code = kErrAltitude;
    else if (!(sun_dec >= -kPi / 2 && sun_dec <= kPi / 2) || !(lat >= -kPi / 2 && lat <= kPi / 2))
        code = kErrAngle;
    else if (d.f10 <= 0.0 || d.f10b <= 0.0 || d.s10 <= 0.0 || d.s10b <= 0.0 || d.m10 <= 0.0 || d.m10b <= 0.0 ||
             d.y10 <= 0.0 || d.y10b <= 0.0)
        code = kErrIndex;
    if (code != 0.0) return code;  // the whole group returns together
    const double alt = alt_m / 1000.0;
    const double fn = fmin(pow(d.f10b / 240.0, 0.25), 1.0);
    const double fsb = d.f10b * fn + d.s10b * (1.0 - fn);
    const double tsubc = 392.4 + 3.227 * fsb + 0.298 * (d.f10 - d.f10b) + 2.259 * (d.s10 - d.s10b) +
                         0.312 * (d.m10 - d.m10b) + 0.178 * (d.y10 - d.y10b);
    const double eta = 0.5 * fabs(lat - sun_dec);
    const double theta = 0.5 * fabs(lat + sun_dec);
    double h = hour_angle;
    if (!(h >= 0.0 && h < kTwoPi)) {
        if (h < 0.0 && h > -kTwoPi) {
            h += kTwoPi;
        } else {
            h = fmod(h, kTwoPi);
            if (h < 0.0) h += kTwoPi;
        }
    }
    const double tau = h - 0.64577182 + 0.10471976 * sin(h + 0.75049158);
    double st_hour = ((h + kPi) * (180.0 / kPi)) / 15.0;
    if (st_hour >= 24.0) st_hour -= 24.0;
    else if (st_hour < 0.0) st_hour += 24.0;
    double slat, clat;
    sincos(lat, &slat, &clat);
    const double cos_eta = five_halves(cos(eta));
    const double sin_theta = five_halves(sin(theta));
    const double cos_tau = fabs(cos(0.5 * tau));
    const double df = sin_theta + (cos_eta - sin_theta) * cos_tau * cos_tau * cos_tau;
    const double tsubl = tsubc * (1.0 + 0.31 * df);
    const double tinf = tsubl + d.dtc + dtc_correction(d.f10, st_hour, clat, alt);
    const double tsubx = 444.3807 + 0.02385 * tinf - 392.8292 * exp(-0.0021357 * tinf);
    const double gsubx = 0.054285714 * (tsubx - 183.0);
    double tc[4];
    tc[0] = tsubx;
    tc[1] = gsubx;
    tc[2] = (tinf - tsubx) / (kPi / 2);
    tc[3] = gsubx / tc[2];
    const double z1 = 90.0;
    double al, zr;
    int n;
    const double mb1 = mbar(z1);
    const double tloc1 = local_temp(z1, tc);
    const bool use_fit = fit_covers(fit, tinf);
    // the 2-D fits need the lower (and, above 500 km, the middle) 1-D fits
    const bool use2 = use_fit && fit2 != nullptr && tinf >= fit2->tlo && tinf <= fit2->thi;
    const double xt2 = use2 ? (2.0 * tinf - (fit2->thi + fit2->tlo)) / (fit2->thi - fit2->tlo) : 0.0;
    SweepG lo;
    double mid_fit_sum = 0.0;  // the middle sweep's fitted sum (used above 500 km)
    if (use_fit && alt >= 105.0) {
        cheb_eval_pair(tinf, &lo.sum, &mid_fit_sum);
        lo.z = fit->low_z;
        lo.zend = fit->low_zend;
        lo.mb = fit->low_mb2;
        lo.gravl = fit->low_gravl;
        lo.tloc = local_temp(lo.z, tc);
    } else {
        al = log(fmin(alt, 105.0) / z1);
        n = 1 + (int)floor(al / kLnStepLower);
        zr = exp(al / n);
        lo = boole_sweep_group<L>(z1, zr, n, mb1 * grav(z1) / tloc1, true, tc, q, gmask);
    }
    const double mb2 = lo.mb, tloc2 = lo.tloc;
    double rho = 3.46e-6 * mb2 * tloc1 / exp(lo.sum / kRstar) / (mb1 * tloc2);
    const double anm = kAvogadro * rho;
    const double an = anm / mb2;
    double fact2 = anm / 28.960;
    const double fac[5] = {JBT(kFrac)[0] * fact2, fact2 * (1.0 + JBT(kFrac)[1]) - an, 2.0 * (an - fact2),
                           JBT(kFrac)[2] * fact2, JBT(kFrac)[3] * fact2};
    double aln[6];
    for (int i = 0; i < 5; ++i) aln[i] = fac[i] < 0.0 ? NAN : log(fac[i]);
    double z = lo.z;
    if (alt <= 105.0) {
        aln[5] = aln[4] - 25.0;
    } else {
        SweepG mid;
        if (use_fit && alt >= 500.0) {
            mid.sum = mid_fit_sum;
            mid.z = fit->mid_z;
            mid.zend = fit->mid_zend;
            mid.tloc = local_temp(mid.z, tc);
            mid.gravl = fit->mid_gravl;
            mid.ain = mid.gravl / mid.tloc;
        } else {
            al = log(fmin(alt, 500.0) / z);
            n = 1 + (int)floor(al / kLnStepMiddle);
            zr = exp(al / n);
            if (use2 && fit2->valid_mid && alt < 500.0 && n >= 1 && n <= kFit2Mid)
                mid = fitted_sweep<L>(&fit2->mid[n - 1][0][0], fit2->mid_ex[n - 1], fit2_x(fit2->mid_rng[n - 1], al),
                                      xt2, lo.zend, zr, n, lo.gravl / tloc2, tc, q, gmask);
            else
                mid = boole_sweep_group<L>(lo.zend, zr, n, lo.gravl / tloc2, false, tc, q, gmask);
        }
        const double tloc3 = mid.tloc;
        z = mid.z;
        al = log(fmax(alt, 500.0) / z);
        const double ustep = alt > 500.0 ? kLnStepUpper : kLnStepMiddle;
        n = 1 + (int)floor(al / ustep);
        zr = exp(al / n);
        SweepG up;
        if (use2 && alt < 500.0 && fit2->valid_uplow && fit2->valid_mid && n >= 1 && n <= kFit2UpLow)
            up = fitted_sweep<L>(&fit2->uplow[n - 1][0][0], fit2->uplow_ex[n - 1],
                                 fit2_x(fit2->uplow_rng[n - 1], al), xt2, mid.zend, zr, n, mid.ain, tc, q, gmask);
        else if (use2 && alt > 500.0 && fit2->valid_uphigh && n >= 1 && n <= kFit2UpHigh)
            up = fitted_sweep<L>(&fit2->uphigh[n - 1][0][0], fit2->uphigh_ex[n - 1],
                                 fit2_x(fit2->uphigh_rng[n - 1], al), xt2, mid.zend, zr, n, mid.ain, tc, q, gmask);
        else
            up = boole_sweep_group<L>(mid.zend, zr, n, mid.ain, false, tc, q, gmask);
        const double tloc4 = up.tloc;
        z = up.z;
        double altr, hsign;
        if (alt <= 500.0) {
            altr = log(tloc3 / tloc2);
            fact2 = mid.sum / kRstar;
            hsign = 1.0;
        } else {
            altr = log(tloc4 / tloc2);
            fact2 = (mid.sum + up.sum) / kRstar;
            hsign = -1.0;
        }
        for (int i = 0; i < 4; ++i) aln[i] = aln[i] - altr - fact2 * JBT(kAmw)[i];
        aln[4] = aln[4] - (1.0 - 0.38) * altr - fact2 * JBT(kAmw)[4];
        const double al10t5 = log10(tinf);
        const double alnh5 = (5.5 * al10t5 - 39.40) * al10t5 + 73.13;
        aln[5] = kLn10 * (alnh5 + 6.0) + hsign * (log(tloc4 / tloc3) + up.sum * JBT(kAmw)[5] / kRstar);
    }
    const double years = (mjd - 36204.0) / 365.2422;
    double capphi = years - trunc(years);
    if (capphi == 0.0) capphi = copysign(0.0, years);
    const double sgn = lat >= 0.0 ? 1.0 : -1.0;
    const double hm90 = alt - 90.0;
    const double dlrsl = 0.02 * hm90 * exp(-0.045 * hm90) * sgn * sin(kTwoPi * capphi + 1.72) * slat * slat;
    double dlrsa = 0.0;
    if (z < 2000.0) {
        bool ok = true;
        const double day = day_of_year(mjd, &ok);
        if (!ok) return kErrDomain;
        const double htz = alt / 1000.0;
        double fsmb = d.f10b - 0.70 * d.s10b - 0.04 * d.m10b;
        const double fzz = JBT(kFzm)[0] + JBT(kFzm)[1] * fsmb + JBT(kFzm)[2] * fsmb * htz +
                           JBT(kFzm)[3] * fsmb * htz * htz + JBT(kFzm)[4] * fsmb * fsmb * htz;
        fsmb = d.f10b - 0.75 * d.s10b - 0.37 * d.m10b;
        double s1, c1;
        sincos(kTwoPi * (day - 1.0) / 365.0, &s1, &c1);
        const double s2 = 2.0 * s1 * c1, c2 = c1 * c1 - s1 * s1;
        const double gtz = JBT(kGtm)[0] + JBT(kGtm)[1] * s1 + JBT(kGtm)[2] * c1 + JBT(kGtm)[3] * s2 +
                           JBT(kGtm)[4] * c2 + JBT(kGtm)[5] * fsmb + JBT(kGtm)[6] * fsmb * s1 +
                           JBT(kGtm)[7] * fsmb * c1 + JBT(kGtm)[8] * fsmb * s2 + JBT(kGtm)[9] * fsmb * c2;
        dlrsa = fmax(fzz, 1.0e-6) * gtz;
    }
    const double dlr = kLn10 * (dlrsl + dlrsa);
    double sumnm = 0.0;
    for (int i = 0; i < 6; ++i) sumnm += exp(aln[i] + dlr) * JBT(kAmw)[i];
    rho = sumnm / kAvogadro;
    double fex = 1.0;
    if (alt >= 1000.0 && alt < 1500.0) {
        const double zeta = (alt - 1000.0) * 0.002;
        const double f15c = JBT(kCht)[0] + JBT(kCht)[1] * d.f10b + JBT(kCht)[2] * 1500.0 +
                            JBT(kCht)[3] * d.f10b * 1500.0;
        const double f15cz = (JBT(kCht)[2] + JBT(kCht)[3] * d.f10b) * 500.0;
        const double fex2 = 3.0 * f15c - f15cz - 3.0;
        const double fex3 = f15cz - 2.0 * f15c + 2.0;
        fex = 1.0 + zeta * zeta * (fex2 + fex3 * zeta);
    } else if (alt >= 1500.0) {
        fex = JBT(kCht)[0] + JBT(kCht)[1] * d.f10b + JBT(kCht)[2] * alt + JBT(kCht)[3] * d.f10b * alt;
    }
    const double out = rho * fex;
    if (!(isfinite(out) && out > 0.0)) return kErrDomain;
    return out;
}
#endif  // __CUDACC__

}  // namespace jb
}  // namespace bqp
