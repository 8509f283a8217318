// Host side of the IAU 2006/2000A frame: the CIO-based GCRS->ITRS chain
// (IERS Conventions 2010, chapter 5; the ERFA/SOFA algorithms the reference
// restates in satpy_core/src/frame_time/) and the 1800 s segment builder of
// the reference's frame authority (authority.rs:488-571).
//
// The chain runs in plain binary64 except where the reference raises it to
// double-double: EOP interpolation of the fixture chain, the Earth rotation
// angle, the outer RPOM * R3(ERA) * RC2I product and the five-point stencil
// (chain.rs, dd.rs, era.rs).  Evaluation order follows the reference's
// sources so that the results agree to the last bits on the same libm.
#include "frame_time_host.h"

#include <algorithm>
#include <atomic>
#include <array>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "iau2000a_tables.h"

namespace bqp {
namespace ft {

namespace {

constexpr double kD2pi = 6.283185307179586476925287;
constexpr double kDas2r = 4.848136811095359935899141e-6;  // arcsec -> rad
constexpr double kTurnas = 1296000.0;
constexpr double kDjc = 36525.0;
constexpr double kDj00 = 2451545.0;
constexpr double kTtmtai = 32.184;
constexpr double kU2r = kDas2r / 1e7;  // 0.1 microarcsec -> rad

// ---------------------------------------------------------- double-double
// Dekker/Knuth pair arithmetic (|lo| <= ulp(hi)/2), in the evaluation order
// of the reference's dd.rs: normalise by fast two-sum, add by two-sum of the
// high parts plus both low parts, multiply with an FMA error term.
struct Dd {
    double hi, lo;
};
inline Dd dd_from(double x) { return {x, 0.0}; }
inline Dd dd_norm(double a, double b) {
    const double s = a + b;
    return {s, b - (s - a)};
}
inline double dd_f64(Dd a) { return a.hi + a.lo; }
inline Dd dd_add(Dd a, Dd b) {
    const double s = a.hi + b.hi;
    const double v = s - a.hi;
    const double e = (a.hi - (s - v)) + (b.hi - v) + a.lo + b.lo;
    return dd_norm(s, e);
}
inline Dd dd_neg(Dd a) { return {-a.hi, -a.lo}; }
inline Dd dd_sub(Dd a, Dd b) { return dd_add(a, dd_neg(b)); }
inline Dd dd_mul(Dd a, Dd b) {
    const double p = a.hi * b.hi;
    const double e = std::fma(a.hi, b.hi, -p) + a.hi * b.lo + a.lo * b.hi;
    return dd_norm(p, e);
}
inline Dd dd_scale(Dd a, double b) { return dd_mul(a, dd_from(b)); }
inline Dd dd_div(Dd a, Dd b) {
    const double q1 = a.hi / b.hi;
    const Dd r = dd_sub(a, dd_mul(b, dd_from(q1)));
    const double q2 = (r.hi + r.lo) / b.hi;
    return dd_add(dd_from(q1), dd_from(q2));
}
// sin/cos of a pair: the low part applied as a first-order correction.
inline void dd_sincos(Dd x, Dd* s_out, Dd* c_out) {
    const double s = std::sin(x.hi), c = std::cos(x.hi);
    *s_out = dd_add(dd_from(s), dd_from(c * x.lo));
    *c_out = dd_sub(dd_from(c), dd_from(s * x.lo));
}

// Earth rotation angle (IERS 2003: 2 pi (0.7790572732640 + 1.00273781191135448
// Tu)), with the two constants and 2 pi as exact pairs of their decimals.
Dd era_dd(Dd u1, Dd u2) {
    const Dd c0{0x1.8ee0984cc2772p-1, 0x1.37791827271b7p-56};
    const Dd c1{0x1.66d9b93e65515p-9, 0x1.1a9fd4c729390p-63};
    const Dd tau{0x1.921fb54442d18p+2, 0x1.1a62633145c07p-52};
    Dd d1 = u1, d2 = u2;
    if (!(dd_f64(u1) < dd_f64(u2))) std::swap(d1, d2);
    const Dd t = dd_add(d1, dd_sub(d2, dd_from(kDj00)));
    const Dd f = dd_add(dd_sub(d1, dd_from(std::floor(d1.hi))), dd_sub(d2, dd_from(std::floor(d2.hi))));
    Dd theta = dd_mul(tau, dd_add(dd_add(f, c0), dd_mul(c1, t)));
    const double turns = std::floor(dd_f64(dd_div(theta, tau)));
    theta = dd_sub(theta, dd_scale(tau, turns));
    if (dd_f64(theta) < 0.0) theta = dd_add(theta, tau);
    return theta;
}

// --------------------------------------------------------------- calendar
// Gregorian date -> MJD (ERFA cal2jd); status 0, -1 bad year, -2 bad month,
// -3 bad day (MJD still formed).
int cal2jd(int iy, int im, int id, double* djm) {
    if (iy < -4799) return -1;
    if (im < 1 || im > 12) return -2;
    static const int mtab[12] = {31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31};
    const int leap = (im == 2 && iy % 4 == 0 && (iy % 100 != 0 || iy % 400 == 0)) ? 1 : 0;
    const int j = (id < 1 || id > mtab[im - 1] + leap) ? -3 : 0;
    const long my = (im - 14) / 12;
    const long iypmy = (long)iy + my;
    *djm = (double)((1461L * (iypmy + 4800L)) / 4L + (367L * (long)(im - 2 - 12 * my)) / 12L -
                    (3L * ((iypmy + 4900L) / 100L)) / 4L + (long)id - 2432076L);
    return j;
}

// Julian day number -> Gregorian date (ERFA jd2cal's integer half).
void jd_to_ymd(int64_t jd, int* iy, int* im, int* id) {
    int64_t l = jd + 68569;
    const int64_t n = (4 * l) / 146097;
    l -= (146097 * n + 3) / 4;
    const int64_t i = (4000 * (l + 1)) / 1461001;
    l -= (1461 * i) / 4 - 31;
    const int64_t k = (80 * l) / 2447;
    *id = (int)(l - (2447 * k) / 80);
    l = k / 11;
    *im = (int)(k + 2 - 12 * l);
    *iy = (int)(100 * (n - 49) + i + l);
}

// TAI - UTC at a date (integer-leap era only: the frame's span starts in
// 1973).  Status 0, or < 0 for a date before 1972 or an invalid date.
int dat(int iy, int im, int id, double fd, double* out) {
    if (!(fd >= 0.0 && fd <= 1.0)) return -4;
    double djm;
    const int j = cal2jd(iy, im, id, &djm);
    if (j < 0) return j;
    const double v = dat_mjd((int32_t)djm);
    if (!(v == v)) return -5;
    *out = v;
    return 0;
}

// UTC calendar instant -> two-part quasi-JD (ERFA dtf2d, scale "UTC"): a day
// that ends in a leap second lasts 86,401 s and accepts 23:59:60.x.
int dtf2d_utc(int iy, int im, int id, int ihr, int imn, double sec, double* d1, double* d2) {
    double w;
    int js = cal2jd(iy, im, id, &w);
    if (js != 0) return js;
    const double dj = kDjm0 + w;
    double day = kDaySec, seclim = 60.0;
    double dat0, dat12, dat24;
    if (dat(iy, im, id, 0.0, &dat0) < 0 || dat(iy, im, id, 0.5, &dat12) < 0) return -5;
    int64_t jdt;
    double fdt;
    if (!jd_split(dj, 1.5, &jdt, &fdt)) return -1;
    int iy2, im2, id2;
    jd_to_ymd(jdt, &iy2, &im2, &id2);
    if (dat(iy2, im2, id2, 0.0, &dat24) < 0) return -5;
    const double dleap = dat24 - (2.0 * dat12 - dat0);
    day += dleap;
    if (ihr == 23 && imn == 59) seclim += dleap;
    if (ihr < 0 || ihr > 23) return -4;
    if (imn < 0 || imn > 59) return -5;
    if (sec < 0.0) return -6;
    js = sec >= seclim ? 2 : 0;
    *d1 = dj;
    *d2 = (60.0 * (double)(60 * ihr + imn) + sec) / day;
    return js;
}

void taitt(double tai1, double tai2, double* tt1, double* tt2) {
    const double dtat = kTtmtai / kDaySec;
    if (std::fabs(tai1) > std::fabs(tai2)) {
        *tt1 = tai1;
        *tt2 = tai2 + dtat;
    } else {
        *tt1 = tai1 + dtat;
        *tt2 = tai2;
    }
}

inline double t_jc(double d1, double d2) { return ((d1 - kDj00) + d2) / kDjc; }

// ------------------------------------------------ fundamental arguments
// IERS Conventions 2003 (MHB2000) polynomials, arcsec and rad.
double fal03(double t) {
    return std::fmod(485868.249036 + t * (1717915923.2178 + t * (31.8792 + t * (0.051635 + t * (-0.00024470)))),
                     kTurnas) * kDas2r;
}
double falp03(double t) {
    return std::fmod(1287104.793048 + t * (129596581.0481 + t * (-0.5532 + t * (0.000136 + t * (-0.00001149)))),
                     kTurnas) * kDas2r;
}
double faf03(double t) {
    return std::fmod(335779.526232 + t * (1739527262.8478 + t * (-12.7512 + t * (-0.001037 + t * (0.00000417)))),
                     kTurnas) * kDas2r;
}
double fad03(double t) {
    return std::fmod(1072260.703692 + t * (1602961601.2090 + t * (-6.3706 + t * (0.006593 + t * (-0.00003169)))),
                     kTurnas) * kDas2r;
}
double faom03(double t) {
    return std::fmod(450160.398036 + t * (-6962890.5431 + t * (7.4722 + t * (0.007702 + t * (-0.00005939)))),
                     kTurnas) * kDas2r;
}
double fame03(double t) { return std::fmod(4.402608842 + 2608.7903141574 * t, kD2pi); }
double fave03(double t) { return std::fmod(3.176146697 + 1021.3285546211 * t, kD2pi); }
double fae03(double t) { return std::fmod(1.753470314 + 628.3075849991 * t, kD2pi); }
double fama03(double t) { return std::fmod(6.203480913 + 334.0612426700 * t, kD2pi); }
double faju03(double t) { return std::fmod(0.599546497 + 52.9690962641 * t, kD2pi); }
double fasa03(double t) { return std::fmod(0.874016757 + 21.3299104960 * t, kD2pi); }
double faur03(double t) { return std::fmod(5.481293872 + 7.4781598567 * t, kD2pi); }
double fapa03(double t) { return (0.024381750 + 0.00000538691 * t) * t; }

}  // namespace

// ---------------------------------------------------------------- nutation
// IAU 2000A nutation (MHB2000): the luni-solar series on the Delaunay
// arguments, then the planetary series on MHB2000's own lunar and planetary
// arguments, each summed from its smallest term up (iau2006.rs:22-105).
void nut00a(double d1, double d2, double* dpsi, double* deps) {
    const double t = t_jc(d1, d2);
    const double el = fal03(t);
    const double elp =
        std::fmod(1287104.79305 + t * (129596581.0481 + t * (-0.5532 + t * (0.000136 + t * (-0.00001149)))),
                  kTurnas) * kDas2r;
    const double f = faf03(t);
    const double d =
        std::fmod(1072260.70369 + t * (1602961601.2090 + t * (-6.3706 + t * (0.006593 + t * (-0.00003169)))),
                  kTurnas) * kDas2r;
    const double om = faom03(t);
    double dp = 0.0, de = 0.0;
    for (int i = iau::kNutLs - 1; i >= 0; --i) {
        const iau::NutLs& x = iau::kNutLsTab[i];
        const double arg = std::fmod((double)x.n[0] * el + (double)x.n[1] * elp + (double)x.n[2] * f +
                                         (double)x.n[3] * d + (double)x.n[4] * om,
                                     kD2pi);
        const double sarg = std::sin(arg), carg = std::cos(arg);
        dp += (x.sp + x.spt * t) * sarg + x.cp * carg;
        de += (x.ce + x.cet * t) * carg + x.se * sarg;
    }
    const double dpsils = dp * kU2r, depsls = de * kU2r;

    const double al = std::fmod(2.35555598 + 8328.6914269554 * t, kD2pi);
    const double af = std::fmod(1.627905234 + 8433.466158131 * t, kD2pi);
    const double ad = std::fmod(5.198466741 + 7771.3771468121 * t, kD2pi);
    const double aom = std::fmod(2.18243920 - 33.757045 * t, kD2pi);
    const double apa = fapa03(t);
    const double alme = fame03(t), alve = fave03(t), alea = fae03(t), alma = fama03(t);
    const double alju = faju03(t), alsa = fasa03(t), alur = faur03(t);
    const double alne = std::fmod(5.321159000 + 3.8127774000 * t, kD2pi);
    dp = 0.0;
    de = 0.0;
    for (int i = iau::kNutPl - 1; i >= 0; --i) {
        const iau::NutPl& x = iau::kNutPlTab[i];
        const double arg = std::fmod(
            (double)x.n[0] * al + (double)x.n[1] * af + (double)x.n[2] * ad + (double)x.n[3] * aom +
                (double)x.n[4] * alme + (double)x.n[5] * alve + (double)x.n[6] * alea + (double)x.n[7] * alma +
                (double)x.n[8] * alju + (double)x.n[9] * alsa + (double)x.n[10] * alur + (double)x.n[11] * alne +
                (double)x.n[12] * apa,
            kD2pi);
        const double sarg = std::sin(arg), carg = std::cos(arg);
        dp += (double)x.sp * sarg + (double)x.cp * carg;
        de += (double)x.se * sarg + (double)x.ce * carg;
    }
    *dpsi = dpsils + dp * kU2r;
    *deps = depsls + de * kU2r;
}

// IAU 2000A nutation adjusted to the IAU 2006 precession (iau2006.rs:107-114).
void nut06a(double d1, double d2, double* dpsi, double* deps) {
    const double t = t_jc(d1, d2);
    const double fj2 = -2.7774e-6 * t;
    double dp, de;
    nut00a(d1, d2, &dp, &de);
    *dpsi = dp + dp * (0.4697e-6 + fj2);
    *deps = de + de * fj2;
}

// Mean obliquity, IAU 2006 (arcsec polynomial).
double obl06(double d1, double d2) {
    const double t = t_jc(d1, d2);
    return (84381.406 +
            (-46.836769 + (-0.0001831 + (0.00200340 + (-0.000000576 + (-0.0000000434) * t) * t) * t) * t) * t) *
           kDas2r;
}

// Fukushima-Williams precession angles, IAU 2006 (iau2006.rs:128-160).
void pfw06(double d1, double d2, double* gamb, double* phib, double* psib, double* epsa) {
    const double t = t_jc(d1, d2);
    *gamb = (-0.052928 +
             (10.556378 + (0.4932044 + (-0.00031238 + (-0.000002788 + (0.0000000260) * t) * t) * t) * t) * t) *
            kDas2r;
    *phib = (84381.412819 +
             (-46.811016 + (0.0511268 + (0.00053289 + (-0.000000440 + (-0.0000000176) * t) * t) * t) * t) * t) *
            kDas2r;
    *psib = (-0.041775 +
             (5038.481484 + (1.5584175 + (-0.00018522 + (-0.000026452 + (-0.0000000148) * t) * t) * t) * t) * t) *
            kDas2r;
    *epsa = obl06(d1, d2);
}

// ----------------------------------------------------------- rotations
static void ident(Mat3 r) {
    for (int i = 0; i < 9; ++i) r[i] = (i % 4 == 0) ? 1.0 : 0.0;
}
// Pre-multiply by R_x(phi), R_y(theta), R_z(psi) (ERFA rx/ry/rz).
static void rx(double phi, Mat3 r) {
    const double s = std::sin(phi), c = std::cos(phi);
    for (int j = 0; j < 3; ++j) {
        const double a1 = c * r[3 + j] + s * r[6 + j];
        const double a2 = -s * r[3 + j] + c * r[6 + j];
        r[3 + j] = a1;
        r[6 + j] = a2;
    }
}
static void ry(double th, Mat3 r) {
    const double s = std::sin(th), c = std::cos(th);
    for (int j = 0; j < 3; ++j) {
        const double a0 = c * r[j] - s * r[6 + j];
        const double a2 = s * r[j] + c * r[6 + j];
        r[j] = a0;
        r[6 + j] = a2;
    }
}
static void rz(double psi, Mat3 r) {
    const double s = std::sin(psi), c = std::cos(psi);
    for (int j = 0; j < 3; ++j) {
        const double a0 = c * r[j] + s * r[3 + j];
        const double a1 = -s * r[j] + c * r[3 + j];
        r[j] = a0;
        r[3 + j] = a1;
    }
}

// Rotation from Fukushima-Williams angles (ERFA fw2m).
static void fw2m(double gamb, double phib, double psi, double eps, Mat3 r) {
    ident(r);
    rz(gamb, r);
    rx(phib, r);
    rz(-psi, r);
    rx(-eps, r);
}

// Bias-precession-nutation matrix, IAU 2006/2000A (iau2006.rs:163-175).
void pnm06a(double d1, double d2, Mat3 r) {
    double gamb, phib, psib, epsa, dp, de;
    pfw06(d1, d2, &gamb, &phib, &psib, &epsa);
    nut06a(d1, d2, &dp, &de);
    fw2m(gamb, phib, psib + dp, epsa + de, r);
}

// CIO locator s given the CIP (x, y), IAU 2006/2000A (iau2006.rs:177-221).
double s06(double d1, double d2, double x, double y) {
    const double t = t_jc(d1, d2);
    const double fa[8] = {fal03(t), falp03(t), faf03(t), fad03(t), faom03(t), fave03(t), fae03(t), fapa03(t)};
    double w0 = 94.00e-6, w1 = 3808.65e-6, w2 = -122.68e-6, w3 = -72574.11e-6, w4 = 27.98e-6;
    const double w5 = 15.62e-6;
    auto acc = [&](double* w, const iau::CioTerm* tab, int n) {
        for (int i = n - 1; i >= 0; --i) {
            double a = 0.0;
            for (int j = 0; j < 8; ++j) a += (double)tab[i].n[j] * fa[j];
            *w += tab[i].s * std::sin(a) + tab[i].c * std::cos(a);
        }
    };
    acc(&w0, iau::kS06S0Tab, iau::kS06S0);
    acc(&w1, iau::kS06S1Tab, iau::kS06S1);
    acc(&w2, iau::kS06S2Tab, iau::kS06S2);
    acc(&w3, iau::kS06S3Tab, iau::kS06S3);
    acc(&w4, iau::kS06S4Tab, iau::kS06S4);
    return (w0 + (w1 + (w2 + (w3 + (w4 + w5 * t) * t) * t) * t) * t) * kDas2r - x * y / 2.0;
}

// CIP X, Y and CIO locator s, IAU 2006/2000A.
void xys06a(double d1, double d2, double* x, double* y, double* s) {
    Mat3 r;
    pnm06a(d1, d2, r);
    *x = r[6];
    *y = r[7];
    *s = s06(d1, d2, *x, *y);
}

// Celestial-to-intermediate matrix from X, Y, s (ERFA c2ixys).
void c2ixys(double x, double y, double s, Mat3 r) {
    const double r2 = x * x + y * y;
    const double e = r2 > 0.0 ? std::atan2(y, x) : 0.0;
    const double d = std::atan(std::sqrt(r2 / (1.0 - r2)));
    ident(r);
    rz(e, r);
    ry(d, r);
    rz(-(e + s), r);
}

// TIO locator s' (ERFA sp00) and the polar-motion matrix (ERFA pom00).
double sp00(double d1, double d2) { return -47e-6 * t_jc(d1, d2) * kDas2r; }
void pom00(double xp, double yp, double sp, Mat3 r) {
    ident(r);
    rz(sp, r);
    ry(-xp, r);
    rx(-yp, r);
}

double era(double u1, double u2) { return dd_f64(era_dd(dd_from(u1), dd_from(u2))); }

int utc_calendar_to_jd(int iy, int im, int id, int ihr, int imn, double sec, double* d1, double* d2) {
    return dtf2d_utc(iy, im, id, ihr, imn, sec, d1, d2);
}

// ------------------------------------------------------------- EOP table
bool Eop::at(int32_t mjd, double out[5]) const {
    if (rec.empty()) {
        for (int i = 0; i < 5; ++i) out[i] = 0.0;
        return true;
    }
    const int64_t i = (int64_t)mjd - first_mjd;
    if (i < 0 || i >= count()) return false;
    for (int q = 0; q < 5; ++q) out[q] = rec[(size_t)i * 5 + q];
    return true;
}

namespace {

// TAI - UTC at 0h UTC of an MJD (eop.rs dat_at_mjd).
bool dat_at_mjd(int32_t mjd, double* out) {
    const double v = dat_mjd(mjd);
    if (!(v == v)) return false;
    *out = v;
    return true;
}

// Four-node Lagrange in pairs (eop.rs lagrange).
Dd lagrange_dd(Dd x, const Dd xs[4], const double ys[4]) {
    Dd sum = dd_from(0.0);
    for (int i = 0; i < 4; ++i) {
        Dd term = dd_from(ys[i]);
        for (int j = 0; j < 4; ++j)
            if (j != i) term = dd_mul(term, dd_div(dd_sub(x, xs[j]), dd_sub(xs[i], xs[j])));
        sum = dd_add(sum, term);
    }
    return sum;
}

typedef Dd DdMat[9];

void dd_matmul(const DdMat a, const DdMat b, DdMat out) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            Dd v = dd_from(0.0);
            for (int k = 0; k < 3; ++k) v = dd_add(v, dd_mul(a[3 * i + k], b[3 * k + j]));
            out[3 * i + j] = v;
        }
}

// The fixture chain's matrix in pairs (chain.rs:140-297).
int frame_matrix_dd(int iy, int im, int id, int ihr, int imn, double sec, int policy, double offset,
                    const Eop& eop, DdMat out) {
    double u1, u2;
    if (dtf2d_utc(iy, im, id, ihr, imn, sec, &u1, &u2) < 0) return -1;
    double a1, a2;
    if (!utc_to_tai(u1, u2, &a1, &a2)) return -2;
    const Dd s1 = dd_from(a1);
    const Dd s2 = dd_add(dd_from(a2), dd_from(offset / kDaySec));
    Dd ut1_tai;
    double xp, yp, dx, dy;
    if (policy == 1) {
        double djm;
        if (cal2jd(iy, im, id, &djm) < 0) return -3;
        const int32_t centre = (int32_t)djm;
        Dd xs[4];
        double raw[4], vx[4], vy[4], vdx[4], vdy[4];
        for (int q = 0; q < 4; ++q) {
            const int32_t mjd = centre - 1 + q;
            double row[5], n1, n2, d;
            if (!eop.at(mjd, row)) return -4;
            if (!utc_to_tai(kDjm0, (double)mjd, &n1, &n2)) return -2;
            xs[q] = dd_scale(dd_add(dd_sub(dd_from(n1), dd_from(a1)), dd_sub(dd_from(n2), dd_from(a2))), kDaySec);
            if (!dat_at_mjd(mjd, &d)) return -2;
            raw[q] = row[2] - d;
            vx[q] = row[0];
            vy[q] = row[1];
            vdx[q] = row[3];
            vdy[q] = row[4];
        }
        const Dd x = dd_from(offset);
        ut1_tai = lagrange_dd(x, xs, raw);
        xp = dd_f64(lagrange_dd(x, xs, vx)) * kDas2r;
        yp = dd_f64(lagrange_dd(x, xs, vy)) * kDas2r;
        dx = dd_f64(lagrange_dd(x, xs, vdx)) * 1e-3 * kDas2r;
        dy = dd_f64(lagrange_dd(x, xs, vdy)) * 1e-3 * kDas2r;
    } else {
        const double fd = ((double)ihr * 3600.0 + (double)imn * 60.0 + std::min(sec, 59.999999)) / kDaySec;
        double d;
        if (dat(iy, im, id, fd, &d) < 0) return -2;
        ut1_tai = dd_from(-d);
        xp = yp = dx = dy = 0.0;
    }
    double tt1, tt2, x, y, s;
    taitt(dd_f64(s1), dd_f64(s2), &tt1, &tt2);
    xys06a(tt1, tt2, &x, &y, &s);
    Mat3 rc2i, rpom;
    c2ixys(x + dx, y + dy, s, rc2i);
    pom00(xp, yp, sp00(tt1, tt2), rpom);
    Dd sn, cs;
    dd_sincos(era_dd(s1, dd_add(s2, dd_div(ut1_tai, dd_from(kDaySec)))), &sn, &cs);
    const Dd z = dd_from(0.0), one = dd_from(1.0);
    const DdMat r3 = {cs, sn, z, dd_neg(sn), cs, z, z, z, one};
    DdMat c_dd, p_dd, mid;
    for (int e = 0; e < 9; ++e) {
        c_dd[e] = dd_from(rc2i[e]);
        p_dd[e] = dd_from(rpom[e]);
    }
    dd_matmul(r3, c_dd, mid);
    dd_matmul(p_dd, mid, out);
    return 0;
}

}  // namespace

int frame_matrix(int iy, int im, int id, int ihr, int imn, double sec, int policy, double offset,
                 const Eop& eop, Mat3 r, double* r_dd) {
    DdMat m;
    const int rc = frame_matrix_dd(iy, im, id, ihr, imn, sec, policy, offset, eop, m);
    if (rc < 0) return rc;
    for (int e = 0; e < 9; ++e) {
        r[e] = dd_f64(m[e]);
        if (r_dd) {
            r_dd[e] = m[e].hi;
            r_dd[9 + e] = m[e].lo;
        }
    }
    return 0;
}

namespace {

// R, Rdot, Rddot in pairs from the centred five-point stencil of step h
// (chain.rs:299-360).
int derivatives_dd(int iy, int im, int id, int ihr, int imn, double sec, int policy, double h, const Eop& eop,
                   DdMat r, DdMat rdot, DdMat rddot) {
    DdMat smp[5];
    for (int q = 0; q < 5; ++q) {
        const int rc = frame_matrix_dd(iy, im, id, ihr, imn, sec, policy, (double)(q - 2) * h, eop, smp[q]);
        if (rc < 0) return rc;
    }
    for (int e = 0; e < 9; ++e) {
        const Dd m2 = smp[0][e], m1 = smp[1][e], v = smp[2][e], p1 = smp[3][e], p2 = smp[4][e];
        const Dd near = dd_sub(p1, m1), far = dd_sub(p2, m2);
        const Dd near2 = dd_add(dd_sub(p1, v), dd_sub(m1, v));
        const Dd far2 = dd_add(dd_sub(p2, v), dd_sub(m2, v));
        r[e] = v;
        rdot[e] = dd_div(dd_sub(dd_scale(near, 8.0), far), dd_from(12.0 * h));
        rddot[e] = dd_div(dd_sub(dd_scale(near2, 16.0), far2), dd_from(12.0 * h * h));
    }
    return 0;
}

}  // namespace

int frame_derivatives(int iy, int im, int id, int ihr, int imn, double sec, int policy, double h,
                      const Eop& eop, Mat3 r, Mat3 rdot, Mat3 rddot) {
    DdMat a, b, c;
    const int rc = derivatives_dd(iy, im, id, ihr, imn, sec, policy, h, eop, a, b, c);
    if (rc < 0) return rc;
    for (int e = 0; e < 9; ++e) {
        r[e] = dd_f64(a[e]);
        rdot[e] = dd_f64(b[e]);
        rddot[e] = dd_f64(c[e]);
    }
    return 0;
}

// A GCRS state (position, velocity, acceleration) in ITRS through R, Rdot
// and Rddot, summed in pairs (chain.rs transform_state):
//   r' = R r,  v' = R v + Rdot r,  a' = R a + 2 Rdot v + Rddot r.
int frame_transform_state(int iy, int im, int id, int ihr, int imn, double sec, int policy, double h,
                          const Eop& eop, const double* r, const double* v, const double* a, double* ro,
                          double* vo, double* ao) {
    DdMat R, Rd, Rdd;
    const int rc = derivatives_dd(iy, im, id, ihr, imn, sec, policy, h, eop, R, Rd, Rdd);
    if (rc < 0) return rc;
    for (int i = 0; i < 3; ++i) {
        Dd p = dd_from(0.0), q = dd_from(0.0), w = dd_from(0.0);
        for (int j = 0; j < 3; ++j) {
            const int e = 3 * i + j;
            p = dd_add(p, dd_scale(R[e], r[j]));
            q = dd_add(q, dd_add(dd_scale(R[e], v[j]), dd_scale(Rd[e], r[j])));
            w = dd_add(w, dd_add(dd_add(dd_scale(R[e], a[j]), dd_scale(Rd[e], 2.0 * v[j])), dd_scale(Rdd[e], r[j])));
        }
        ro[i] = dd_f64(p);
        vo[i] = dd_f64(q);
        ao[i] = dd_f64(w);
    }
    return 0;
}

// ------------------------------------------------------------- authority
namespace {

// TAI seconds of a node's 0h UTC and its TAI - UTC (authority.rs:900-923).
bool node_tai(int32_t mjd, double* tai, double* delta_at) {
    if (!dat_at_mjd(mjd, delta_at)) return false;
    *tai = (double)(mjd - kOriginMjd) * kDaySec + *delta_at;
    return true;
}

// Two-part TAI JD of a continuous-TAI instant (authority.rs:1063-1076).
void tai_jd(double tai_s, double* jd1, double* jd2) {
    double day = std::floor(tai_s / kDaySec);
    double frac = tai_s - day * kDaySec;
    if (frac < 0.0) {
        day -= 1.0;
        frac += kDaySec;
    } else if (frac >= kDaySec) {
        day += 1.0;
        frac -= kDaySec;
    }
    *jd1 = kDjm0 + (double)kOriginMjd + day;
    *jd2 = frac / kDaySec;
}

double lagrange4(const double v[4], const double a[4]) {
    double t[4];
    for (int i = 0; i < 4; ++i) {
        t[i] = v[i];
        for (int j = 0; j < 4; ++j)
            if (j != i) t[i] *= (0.0 - a[j]) / (a[i] - a[j]);
    }
    double s = 0.0;
    for (int i = 0; i < 4; ++i) s += t[i];
    return s;
}

struct EopAt {
    double xp, yp, dx, dy, ut1_tai, jd1, jd2;
};

// Bulletin-A quantities at an instant: four-node Lagrange in continuous TAI
// over the days centre-1 .. centre+2, UT1 - TAI with each node's own
// TAI - UTC removed (authority.rs:925-1022).
bool eop_at(const Eop& eop, double tai_s, double delta_at, EopAt* o) {
    const double utc_mjd = (tai_s - delta_at) / kDaySec + (double)kOriginMjd;
    const double cf = std::floor(utc_mjd);
    if (!(cf > -2.0e9 && cf < 2.0e9)) return false;
    const int32_t centre = (int32_t)cf;
    tai_jd(tai_s, &o->jd1, &o->jd2);
    double ab[4], x[4], y[4], dxv[4], dyv[4], u[4];
    for (int q = 0; q < 4; ++q) {
        const int32_t mjd = centre - 1 + q;
        double row[5], nt, nd;
        if (!eop.at(mjd, row) || !node_tai(mjd, &nt, &nd)) return false;
        ab[q] = nt - tai_s;
        x[q] = row[0];
        y[q] = row[1];
        u[q] = row[2] - nd;
        dxv[q] = row[3];
        dyv[q] = row[4];
    }
    o->xp = lagrange4(x, ab) * kDas2r;
    o->yp = lagrange4(y, ab) * kDas2r;
    o->dx = lagrange4(dxv, ab) * 1e-3 * kDas2r;
    o->dy = lagrange4(dyv, ab) * 1e-3 * kDas2r;
    o->ut1_tai = lagrange4(u, ab);
    return true;
}

void matmul3(const double* a, const double* b, double* o) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            o[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
}

// RPOM E_i RC2I for the three selectors E1 = diag(1,1,0), E2 = [[0,1,0],
// [-1,0,0],[0,0,0]], E3 = diag(0,0,1) (authority.rs:343-353), and the ERA
// at the same instant (authority.rs:1078-1107).
bool split_at(const Eop& eop, double tai_s, double delta_at, double m[3][9]) {
    EopAt e;
    if (!eop_at(eop, tai_s, delta_at, &e)) return false;
    double tt1, tt2, x, y, s;
    taitt(e.jd1, e.jd2, &tt1, &tt2);
    xys06a(tt1, tt2, &x, &y, &s);
    Mat3 rc2i, rpom;
    c2ixys(x + e.dx, y + e.dy, s, rc2i);
    pom00(e.xp, e.yp, sp00(tt1, tt2), rpom);
    static const double E[3][9] = {{1, 0, 0, 0, 1, 0, 0, 0, 0}, {0, 1, 0, -1, 0, 0, 0, 0, 0}, {0, 0, 0, 0, 0, 0, 0, 0, 1}};
    for (int i = 0; i < 3; ++i) {
        double t[9];
        matmul3(E[i], rc2i, t);
        matmul3(rpom, t, m[i]);
    }
    return true;
}

bool theta_at(const Eop& eop, double tai_s, double delta_at, double* theta) {
    EopAt e;
    if (!eop_at(eop, tai_s, delta_at, &e)) return false;
    *theta = dd_f64(era_dd(dd_from(e.jd1), dd_add(dd_from(e.jd2), dd_from(e.ut1_tai / kDaySec))));
    return true;
}

// Onto the 2 pi branch of `ref` (authority.rs:1109-1111).
double unwrap_near(double theta, double ref) { return theta + kD2pi * std::round((ref - theta) / kD2pi); }

}  // namespace

Authority::Authority(const Eop& eop) : eop_(eop) {
    // Leap intervals over the span: from the origin to the table's last day,
    // or to 2050-01-01 with zero EOP (authority.rs:192-220).
    const int32_t last = eop_.rec.empty() ? 69806 : eop_.first_mjd + eop_.count() - 1;
    std::memset(&ivl_, 0, sizeof(ivl_));
    double prev = NAN;
    for (int32_t mjd = kOriginMjd; mjd <= last; ++mjd) {
        const double d = dat_mjd(mjd);
        if (!(d == d) || d == prev) continue;
        if (ivl_.n < kMaxIntervals) {
            ivl_.start[ivl_.n] = (double)(mjd - kOriginMjd) * kDaySec + d;
            ivl_.delta_at[ivl_.n] = d;
            ++ivl_.n;
        }
        prev = d;
    }
    double end, d;
    ivl_.span_end = node_tai(last + 1, &end, &d) ? end : 0.0;
}

bool Authority::build(int32_t j, int64_t k, FrameSeg* out) const {
    if (j < 0 || j >= ivl_.n || k < 0) return false;
    const double start = ivl_.start[j], delta_at = ivl_.delta_at[j];
    const double centre = start + ((double)k + 0.5) * kSegWidth;
    const double half = kSegWidth / 2.0;
    double th_c, th_m, th_p;
    if (!theta_at(eop_, centre, delta_at, &th_c) || !theta_at(eop_, centre - half, delta_at, &th_m) ||
        !theta_at(eop_, centre + half, delta_at, &th_p))
        return false;
    th_m = unwrap_near(th_m, th_c);
    th_p = unwrap_near(th_p, th_c);
    double mc[3][9], mm[3][9], mp[3][9];
    if (!split_at(eop_, centre, delta_at, mc) || !split_at(eop_, centre - half, delta_at, mm) ||
        !split_at(eop_, centre + half, delta_at, mp))
        return false;
    for (int i = 0; i < 3; ++i)
        for (int e = 0; e < 9; ++e) {
            out->m[i][e] = mc[i][e];
            out->k[i][e] = (mp[i][e] - mm[i][e]) / (2.0 * half);
        }
    out->b[0] = th_c;
    out->b[1] = (th_p - th_m) / (2.0 * half);
    out->b[2] = (th_p - 2.0 * th_c + th_m) / (2.0 * half * half);
    out->b[3] = 0.0;
    out->centre = centre;
    out->delta_at = delta_at;
    return true;
}

void Authority::keys_between(double lo, double hi, std::vector<std::pair<int32_t, int64_t>>* out) const {
    int32_t j0, j1;
    int64_t k0, k1;
    if (!(lo <= hi)) return;
    lo = std::max(lo, ivl_.n > 0 ? ivl_.start[0] : lo);
    hi = std::min(hi, std::nextafter(ivl_.span_end, -INFINITY));
    if (!segment_index(ivl_, lo, &j0, &k0) || !segment_index(ivl_, hi, &j1, &k1)) return;
    for (int32_t j = j0; j <= j1; ++j) {
        const int64_t ka = j == j0 ? k0 : 0;
        int64_t kb;
        if (j == j1) {
            kb = k1;
        } else {
            const int64_t whole = (int64_t)std::floor((ivl_.start[j + 1] - ivl_.start[j]) / kSegWidth);
            kb = std::max<int64_t>(whole - 1, 0);
        }
        for (int64_t k = ka; k <= kb; ++k) out->push_back({j, k});
    }
}

bool Authority::segment(double tai, int64_t* key, FrameSeg* out) {
    int32_t j;
    int64_t k;
    if (!segment_index(ivl_, tai, &j, &k)) return false;
    std::vector<int64_t> keys;
    std::vector<FrameSeg> segs;
    ensure({{j, k}}, &keys, &segs);
    if (keys.empty()) return false;
    *key = keys[0];
    *out = segs[0];
    return true;
}

void Authority::ensure(const std::vector<std::pair<int32_t, int64_t>>& want, std::vector<int64_t>* built_keys,
                       std::vector<FrameSeg>* built) {
    std::vector<std::pair<int32_t, int64_t>> todo;
    {
        std::lock_guard<std::mutex> g(mu_);
        for (const auto& jk : want) {
            const int64_t key = seg_key(jk.first, jk.second);
            if (!cache_.count(key) && !failed_.count(key)) todo.push_back(jk);
        }
    }
    if (!todo.empty()) {
        std::vector<FrameSeg> segs(todo.size());
        std::vector<char> ok(todo.size(), 0);
        const size_t nt = std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()),
                                           std::max<size_t>(1, todo.size() / 8));
        // workers take segments from a shared counter; the calling thread
        // works too, so a thread that cannot be started costs only speed
        std::atomic<size_t> next{0};
        auto work = [&]() {
            for (size_t i; (i = next.fetch_add(1)) < todo.size();)
                ok[i] = build(todo[i].first, todo[i].second, &segs[i]);
        };
        std::vector<std::thread> th;
        for (size_t w = 1; w < nt; ++w) {
            try {
                th.emplace_back(work);
            } catch (...) {
                break;
            }
        }
        work();
        for (auto& t : th) t.join();
        std::lock_guard<std::mutex> g(mu_);
        for (size_t i = 0; i < todo.size(); ++i) {
            const int64_t key = seg_key(todo[i].first, todo[i].second);
            if (ok[i]) cache_[key] = segs[i];
            else failed_[key] = true;
        }
    }
    std::lock_guard<std::mutex> g(mu_);
    std::vector<int64_t> keys;
    for (const auto& jk : want) keys.push_back(seg_key(jk.first, jk.second));
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    built_keys->clear();
    built->clear();
    for (int64_t key : keys) {
        auto it = cache_.find(key);
        if (it == cache_.end()) continue;
        built_keys->push_back(key);
        built->push_back(it->second);
    }
}

}  // namespace ft
}  // namespace bqp

// ----------------------------------------------------------------- C ABI
// Primitives of the chain, for callers that check it piece by piece.
using namespace bqp::ft;

extern "C" {

void bqp_frame_nut(double d1, double d2, int32_t iau2006, double* out) {
    if (iau2006) nut06a(d1, d2, &out[0], &out[1]);
    else nut00a(d1, d2, &out[0], &out[1]);
}
double bqp_frame_obl06(double d1, double d2) { return obl06(d1, d2); }
void bqp_frame_pfw06(double d1, double d2, double* out) { pfw06(d1, d2, &out[0], &out[1], &out[2], &out[3]); }
void bqp_frame_xys06a(double d1, double d2, double* out) { xys06a(d1, d2, &out[0], &out[1], &out[2]); }
void bqp_frame_c2ixys(double x, double y, double s, double* r) { c2ixys(x, y, s, r); }
double bqp_frame_sp00(double d1, double d2) { return sp00(d1, d2); }
void bqp_frame_pom00(double xp, double yp, double sp, double* r) { pom00(xp, yp, sp, r); }
double bqp_frame_era(double u1, double u2) { return era(u1, u2); }

int bqp_frame_utc_calendar(int32_t y, int32_t m, int32_t d, int32_t hh, int32_t mm, double ss, double* out) {
    return utc_calendar_to_jd(y, m, d, hh, mm, ss, &out[0], &out[1]) < 0 ? -1 : 0;
}

// utc_jd2 null: one-part Julian days in utc_jd.
int bqp_frame_tai_seconds(int64_t n, const double* utc_jd, const double* utc_jd2, double* tai_s) {
    if (n < 0 || (n > 0 && (!utc_jd || !tai_s))) return -1;
    int bad = 0;
    for (int64_t i = 0; i < n; ++i)
        if (!(utc_jd2 ? tai_seconds_from_utc_parts(utc_jd[i], utc_jd2[i], &tai_s[i])
                      : tai_seconds_from_utc_jd(utc_jd[i], &tai_s[i]))) {
            tai_s[i] = NAN;
            bad = 1;
        }
    return bad ? 1 : 0;
}

static Eop make_eop(const double* eop, int32_t first_mjd, int32_t n) {
    Eop e;
    if (eop && n > 0) {
        e.first_mjd = first_mjd;
        e.rec.assign(eop, eop + (size_t)n * 5);
    }
    return e;
}

int bqp_frame_matrix(int32_t y, int32_t m, int32_t d, int32_t hh, int32_t mm, double ss, int32_t policy,
                     double offset, const double* eop, int32_t first_mjd, int32_t n_eop, double* r) {
    if (!r || (policy != 0 && policy != 1)) return -1;
    try {
        return frame_matrix(y, m, d, hh, mm, ss, policy, offset, make_eop(eop, first_mjd, n_eop), r, nullptr);
    } catch (...) {
        return -5;
    }
}

int bqp_frame_transform_state(int32_t y, int32_t m, int32_t d, int32_t hh, int32_t mm, double ss, int32_t policy,
                              double h, const double* eop, int32_t first_mjd, int32_t n_eop, const double* r,
                              const double* v, const double* a, double* r_out, double* v_out, double* a_out) {
    if (!r || !v || !a || !r_out || !v_out || !a_out || (policy != 0 && policy != 1) || !(h > 0.0)) return -1;
    try {
        return frame_transform_state(y, m, d, hh, mm, ss, policy, h, make_eop(eop, first_mjd, n_eop), r, v, a,
                                     r_out, v_out, a_out);
    } catch (...) {
        return -5;
    }
}

int bqp_frame_derivatives(int32_t y, int32_t m, int32_t d, int32_t hh, int32_t mm, double ss, int32_t policy,
                          double h, const double* eop, int32_t first_mjd, int32_t n_eop, double* r, double* rdot,
                          double* rddot) {
    if (!r || !rdot || !rddot || (policy != 0 && policy != 1) || !(h > 0.0)) return -1;
    try {
        return frame_derivatives(y, m, d, hh, mm, ss, policy, h, make_eop(eop, first_mjd, n_eop), r, rdot, rddot);
    } catch (...) {
        return -5;
    }
}

}  // extern "C"

// A standalone segment authority over an EOP table (or zero EOP), for
// callers that evaluate the frame on the host or hand its segments on.
struct bqp_frame_authority {
    Authority a;
    explicit bqp_frame_authority(const Eop& e) : a(e) {}
};

extern "C" {

bqp_frame_authority* bqp_frame_authority_new(const double* eop, int32_t first_mjd, int32_t n_eop) {
    if (n_eop < 0 || (n_eop > 0 && !eop)) return nullptr;
    try {
        return new bqp_frame_authority(make_eop(eop, first_mjd, n_eop));
    } catch (...) {
        return nullptr;
    }
}

void bqp_frame_authority_free(bqp_frame_authority* h) { delete h; }

// Leap intervals: out[0] = n, out[1..48] starts, out[49..96] TAI - UTC,
// out[97] the span's exclusive end.
int bqp_frame_authority_intervals(const bqp_frame_authority* h, double* out) {
    if (!h || !out) return -1;
    const FrameIntervals& I = h->a.intervals();
    out[0] = I.n;
    for (int i = 0; i < kMaxIntervals; ++i) {
        out[1 + i] = I.start[i];
        out[1 + kMaxIntervals + i] = I.delta_at[i];
    }
    out[1 + 2 * kMaxIntervals] = I.span_end;
    return 0;
}

// R [n][9] and w [n][3] at continuous-TAI instants; rows outside the span
// (or whose segment does not build) get NaN and make the return 1.
int bqp_frame_authority_rotation(bqp_frame_authority* h, int64_t n, const double* tai, double* r, double* w) {
    if (!h || n < 0 || (n > 0 && (!tai || !r || !w))) return -1;
    try {
        int bad = 0;
        for (int64_t i = 0; i < n; ++i) {
            FrameSeg s;
            int64_t key;
            if (!h->a.segment(tai[i], &key, &s)) {
                for (int e = 0; e < 9; ++e) r[i * 9 + e] = NAN;
                for (int e = 0; e < 3; ++e) w[i * 3 + e] = NAN;
                bad = 1;
                continue;
            }
            FrameRot fr;
            rotation_at(s, tai[i], fr);
            for (int e = 0; e < 9; ++e) r[i * 9 + e] = fr.r[e];
            for (int e = 0; e < 3; ++e) w[i * 3 + e] = fr.w[e];
        }
        return bad;
    } catch (...) {
        return -5;
    }
}

// The segments holding [lo, hi]: keys [cap] and segments [cap][60] (M0..M2,
// K0..K2 row-major, b0..b3, centre, TAI - UTC).  Returns how many, or -1
// when `cap` is too small (nothing written).
int64_t bqp_frame_authority_segments(bqp_frame_authority* h, double lo, double hi, int64_t cap, int64_t* keys,
                                     double* segs) {
    if (!h || cap < 0) return -1;
    try {
        std::vector<std::pair<int32_t, int64_t>> want;
        h->a.keys_between(lo, hi, &want);
        std::vector<int64_t> k;
        std::vector<FrameSeg> s;
        h->a.ensure(want, &k, &s);
        if ((int64_t)k.size() > cap || (!k.empty() && (!keys || !segs))) return -1;
        static_assert(sizeof(FrameSeg) == 60 * sizeof(double), "segment layout");
        for (size_t i = 0; i < k.size(); ++i) {
            keys[i] = k[i];
            std::memcpy(segs + i * 60, &s[i], sizeof(FrameSeg));
        }
        return (int64_t)k.size();
    } catch (...) {
        return -5;
    }
}

}  // extern "C"

// ------------------------------------------------------ IERS finals text
// Earth-orientation records from IERS finals2000A text, by the reference's
// column rules (frame_time/eop.rs load_eop): lines of at least 125
// characters, MJD in columns 7..15, the three I/P flags at 16, 57 and 95,
// x_p 18..27 and y_p 37..46 (arcsec), UT1-UTC 58..68 (s), dX 97..106 and
// dY 116..125 (mas).  Rows whose flags or fields fail are skipped; the
// table is the contiguous run of days from the first complete one.
namespace {
bool fixed_field(const char* line, int start, int width, double* out) {
    char buf[32];
    int a = start, b = start + width;
    while (a < b && line[a] == ' ') ++a;
    while (b > a && line[b - 1] == ' ') --b;
    if (b <= a || b - a >= (int)sizeof(buf)) return false;
    std::memcpy(buf, line + a, (size_t)(b - a));
    buf[b - a] = '\0';
    char* end = nullptr;
    const double v = std::strtod(buf, &end);
    if (end != buf + (b - a) || !std::isfinite(v)) return false;
    *out = v;
    return true;
}
}  // namespace

extern "C" int64_t bqp_frame_eop_from_finals(const char* text, int64_t len, int64_t cap, int32_t* first_mjd,
                                             double* records) {
    if (!text || len < 0 || !first_mjd) return -1;
    try {
        std::map<int32_t, std::array<double, 5>> rows;
        int64_t pos = 0;
        while (pos < len) {
            int64_t end = pos;
            while (end < len && text[end] != '\n') ++end;
            const int64_t n = end - pos - ((end > pos && text[end - 1] == '\r') ? 1 : 0);
            if (n >= 125) {
                const char* ln = text + pos;
                double mjd, v[5];
                const bool flags = (ln[16] == 'I' || ln[16] == 'P') && (ln[57] == 'I' || ln[57] == 'P') &&
                                   (ln[95] == 'I' || ln[95] == 'P');
                if (flags && fixed_field(ln, 7, 8, &mjd) && mjd == std::floor(mjd) && fixed_field(ln, 18, 9, &v[0]) &&
                    fixed_field(ln, 37, 9, &v[1]) && fixed_field(ln, 58, 10, &v[2]) && fixed_field(ln, 97, 9, &v[3]) &&
                    fixed_field(ln, 116, 9, &v[4])) {
                    const int32_t m = (int32_t)mjd;
                    if (rows.count(m)) return -3;  // a day given twice
                    rows[m] = {v[0], v[1], v[2], v[3], v[4]};
                }
            }
            pos = end + 1;
        }
        if (rows.empty()) return 0;
        const int32_t first = rows.begin()->first;
        int64_t count = 0;
        for (auto it = rows.begin(); it != rows.end() && it->first == first + count; ++it) ++count;
        *first_mjd = first;
        if (!records || cap < count) return count;
        int64_t i = 0;
        for (auto it = rows.begin(); i < count; ++it, ++i)
            for (int q = 0; q < 5; ++q) records[i * 5 + q] = it->second[q];
        return count;
    } catch (...) {
        return -5;
    }
}
