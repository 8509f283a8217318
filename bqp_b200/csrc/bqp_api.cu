// Host side of libbqp_b200.so: the C ABI declared in include/bqp_prop.h.
//
// A context owns the device copy of the gravity table (normalised, with the
// recursion coefficients and the folded summation weights per V/W cell), the
// force/solver configuration, a device work-queue counter and a growable
// device workspace for the host-buffer entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/bqp_prop.h"
#include "launch.h"
#include "frame_time_host.h"
#include "eclipse.cuh"
#include "ephemeris.h"
#include "space_weather.h"
#include "surrogate.h"

using namespace bqp;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(BQP_E_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

constexpr int kMaxOrder = 128;
constexpr size_t kSmemLimit = 227 * 1024;

// Normalised coefficients, [n*(order+1) + m].
struct Coeffs {
    int order = 0;
    std::vector<double> c, s;
};

// "deg ord C S" text, normalised (lightyear_odeint_rs/src/config.rs:128-225):
// blank and '#' lines skipped, lines with fewer than four fields skipped,
// D/d exponents accepted, rows above the requested order ignored.
bool parse_coeffs(const char* text, int64_t len, int order, Coeffs& out, std::string& why) {
    out.order = order;
    out.c.assign((size_t)(order + 1) * (order + 1), 0.0);
    out.s.assign((size_t)(order + 1) * (order + 1), 0.0);
    std::string all(text, (size_t)len);
    std::istringstream in(all);
    std::string line;
    int lineno = 0;
    while (std::getline(in, line)) {
        ++lineno;
        size_t a = line.find_first_not_of(" \t\r");
        if (a == std::string::npos || line[a] == '#') continue;
        std::istringstream ls(line);
        std::string f[4];
        if (!(ls >> f[0] >> f[1] >> f[2] >> f[3])) continue;
        for (int i = 2; i < 4; ++i)
            for (auto& ch : f[i])
                if (ch == 'D' || ch == 'd') ch = 'E';
        char* end = nullptr;
        long deg = std::strtol(f[0].c_str(), &end, 10);
        if (*end || deg < 0) { why = "bad degree on line " + std::to_string(lineno); return false; }
        long m = std::strtol(f[1].c_str(), &end, 10);
        if (*end || m < 0) { why = "bad order on line " + std::to_string(lineno); return false; }
        double cv = std::strtod(f[2].c_str(), &end);
        if (*end || !std::isfinite(cv)) { why = "bad C value on line " + std::to_string(lineno); return false; }
        double sv = std::strtod(f[3].c_str(), &end);
        if (*end || !std::isfinite(sv)) { why = "bad S value on line " + std::to_string(lineno); return false; }
        if (deg <= order && m <= deg) {
            out.c[(size_t)deg * (order + 1) + m] = cv;
            out.s[(size_t)deg * (order + 1) + m] = sv;
        }
    }
    return true;
}

// Per-cell table of the normalised column recursion (see gravity.cuh).  The
// C00 term is left out: the propagator removes the central term analytically
// (rhs.rs:2735-2744, 2849-2855), which is what dropping it computes exactly.
std::vector<double> build_gravity_table(const Coeffs& cf, int order) {
    typedef long double LD;
    const int N = order;
    const int ncells = gravity_cells(N);
    std::vector<double> tab((size_t)ncells * kCellDoubles, 0.0);
    const int ld = cf.order + 1;
    auto C = [&](int n, int k) -> LD {
        if (n < 0 || k < 0 || k > n || n > N) return 0.0L;
        if (n == 0) return 0.0L;  // central term handled analytically
        return (LD)cf.c[(size_t)n * ld + k];
    };
    auto S = [&](int n, int k) -> LD {
        if (n < 0 || k < 0 || k > n || n > N) return 0.0L;
        return (LD)cf.s[(size_t)n * ld + k];
    };
    // N(n,k)/N(n+1,k+1), N(n,k)/N(n+1,k-1), N(n,k)/N(n+1,k)
    auto r_up = [](int n, int k) -> LD {
        LD d = (k == 0) ? 1.0L : 2.0L;
        return std::sqrt(d * (2.0L * n + 1) * (LD)(n + k + 2) * (LD)(n + k + 1) / (2.0L * (2.0L * n + 3)));
    };
    auto r_dn = [](int n, int k) -> LD {
        LD d = (k - 1 == 0) ? 1.0L : 2.0L;
        return std::sqrt(2.0L * (2.0L * n + 1) / (d * (2.0L * n + 3) * (LD)(n - k + 2) * (LD)(n - k + 1)));
    };
    auto r_eq = [](int n, int k) -> LD {
        return std::sqrt((2.0L * n + 1) * (LD)(n + k + 1) / ((2.0L * n + 3) * (LD)(n - k + 1)));
    };
    const LD gm_r2 = (LD)kMu / ((LD)kReGravity * (LD)kReGravity);
    size_t cell = 0;
    for (int j = 0; j <= N + 1; ++j) {
        for (int l = j; l <= N + 1; ++l, ++cell) {
            double* o = &tab[cell * kCellDoubles];
            LD a = 0.0L, b = 0.0L;
            if (l == j) {
                a = (j == 0) ? 0.0L : (j == 1 ? std::sqrt(3.0L) : std::sqrt((2.0L * j + 1) / (2.0L * j)));
            } else if (l == j + 1) {
                a = std::sqrt(2.0L * j + 3);
            } else {
                a = std::sqrt((2.0L * l - 1) * (2.0L * l + 1) / ((LD)(l - j) * (LD)(l + j)));
                b = std::sqrt((2.0L * l + 1) * (LD)(l + j - 1) * (LD)(l - j - 1) /
                              ((2.0L * l - 3) * (LD)(l + j) * (LD)(l - j)));
            }
            const int n = l - 1;
            LD Ax = 0, Bx = 0, Ay = 0, By = 0, Az = 0, Bz = 0;
            if (n >= 0) {
                if (j == 1) {
                    const LD cu = C(n, 0) * r_up(n, 0);
                    Ax += -cu;
                    By += -cu;
                } else if (j >= 2) {
                    const LD r = r_up(n, j - 1);
                    const LD cu = C(n, j - 1) * r, su = S(n, j - 1) * r;
                    Ax += -0.5L * cu;
                    Bx += -0.5L * su;
                    Ay += 0.5L * su;
                    By += -0.5L * cu;
                }
                if (j + 1 <= n) {
                    const int k = j + 1;
                    const LD f = (LD)(n - k + 2) * (LD)(n - k + 1);
                    const LD r = r_dn(n, k);
                    const LD cu = C(n, k) * r, su = S(n, k) * r;
                    Ax += 0.5L * f * cu;
                    Bx += 0.5L * f * su;
                    Ay += 0.5L * f * su;
                    By += -0.5L * f * cu;
                }
                if (j <= n) {
                    const LD r = r_eq(n, j);
                    const LD w = (LD)(n - j + 1);
                    Az += -w * C(n, j) * r;
                    Bz += -w * S(n, j) * r;
                }
            }
            o[0] = (double)a;
            o[1] = (double)b;
            o[2] = (double)(Ax * gm_r2);
            o[3] = (double)(Bx * gm_r2);
            o[4] = (double)(Ay * gm_r2);
            o[5] = (double)(By * gm_r2);
            o[6] = (double)(Az * gm_r2);
            o[7] = (double)(Bz * gm_r2);
        }
    }
    return tab;
}

// Chebyshev fits of the JB2008 fixed-node sweeps (jb2008.cuh, JbFit): the
// sums are evaluated by the quadrature itself at 64 Chebyshev points of
// T_inf in [300, 3500] K, transformed in long double, and checked at 257
// further points; a fit that misses 4e-15 relative is not used.
void sweep_sums(double tinf, jb::Sweep* lo_out, jb::Sweep* mid_out) {
    using namespace jb;
    const double tsubx = 444.3807 + 0.02385 * tinf - 392.8292 * std::exp(-0.0021357 * tinf);
    const double gsubx = 0.054285714 * (tsubx - 183.0);
    double tc[4] = {tsubx, gsubx, (tinf - tsubx) / (kPi / 2), 0.0};
    tc[3] = gsubx / tc[2];
    const double z1 = 90.0;
    double al = std::log(105.0 / z1);
    int n = 1 + (int)std::floor(al / kLnStepLower);
    double zr = std::exp(al / n);
    const double tloc1 = local_temp(z1, tc);
    *lo_out = boole_sweep(z1, z1, zr, n, mbar(z1) * grav(z1) / tloc1, true, tc);
    const double z = lo_out->z;
    al = std::log(500.0 / z);
    n = 1 + (int)std::floor(al / kLnStepMiddle);
    zr = std::exp(al / n);
    *mid_out = boole_sweep(z, lo_out->zend, zr, n, lo_out->gravl / lo_out->tloc, false, tc);
}

// 2-D fits of the altitude-dependent sweeps (jb2008.cuh, JbFit2), for the
// T_inf range the context's drivers can produce.  Each segment's series is
// sampled at Chebyshev points of its reachable log-ratio range and of T_inf
// (the quadrature itself, as the device would walk it), transformed, and
// checked at interior points off the sampling grid; a family whose worst
// error exceeds 1e-13 of max(|sum|, 1) is switched off.
namespace fit2 {

struct Temp {
    double tc[4];
};
Temp temp_profile(double tinf) {
    Temp t;
    const double tsubx = 444.3807 + 0.02385 * tinf - 392.8292 * std::exp(-0.0021357 * tinf);
    const double gsubx = 0.054285714 * (tsubx - 183.0);
    t.tc[0] = tsubx;
    t.tc[1] = gsubx;
    t.tc[2] = (tinf - tsubx) / (kPi / 2);
    t.tc[3] = gsubx / t.tc[2];
    return t;
}

// T_inf bounds for fixed drivers: the diurnal / latitude factor df spans
// [0, 1] and the local-time / latitude / altitude temperature correction is
// bounded on a fine grid.
void tinf_range(const jb::Drivers& d, double* lo, double* hi) {
    const double fn = std::fmin(std::pow(d.f10b / 240.0, 0.25), 1.0);
    const double fsb = d.f10b * fn + d.s10b * (1.0 - fn);
    const double tsubc = 392.4 + 3.227 * fsb + 0.298 * (d.f10 - d.f10b) + 2.259 * (d.s10 - d.s10b) +
                         0.312 * (d.m10 - d.m10b) + 0.178 * (d.y10 - d.y10b);
    double cmin = 1e300, cmax = -1e300;
    for (int ih = 0; ih <= 480; ++ih)
        for (int ic = 0; ic <= 50; ++ic)
            for (int ia = 0; ia <= 60; ++ia) {
                const double v = jb::dtc_correction(d.f10, ih * 0.05, ic * 0.02, 90.0 + ia * 50.0);
                cmin = std::fmin(cmin, v);
                cmax = std::fmax(cmax, v);
            }
    *lo = std::fmin(tsubc, tsubc * 1.31) + d.dtc + cmin - 10.0;
    *hi = std::fmax(tsubc, tsubc * 1.31) + d.dtc + cmax + 10.0;
}

enum Family { kMid = 0, kUpLow = 1, kUpHigh = 2 };

// Where a family's sweep starts and how it is cut, at log-ratio al.
struct Geometry {
    double zend_start, zr;
    int n;
    double ain_z;  // altitude whose g/T is carried into interval 0
};
// n_force > 0 fixes the sweep's interval count (a segment's ends belong to
// its own count, though floor() at the upper end gives the next one).
Geometry geometry(Family fam, const jb::JbFit& f1, double al, int n_force = 0) {
    using namespace jb;
    Geometry g{};
    if (fam == kMid) {
        g.n = n_force > 0 ? n_force : 1 + (int)std::floor(al / kLnStepMiddle);
        g.zr = std::exp(al / g.n);
        g.zend_start = f1.low_zend;
        g.ain_z = f1.low_z;
    } else if (fam == kUpHigh) {
        g.n = n_force > 0 ? n_force : 1 + (int)std::floor(al / kLnStepUpper);
        g.zr = std::exp(al / g.n);
        g.zend_start = f1.mid_zend;
        g.ain_z = f1.mid_z;
    } else {
        // the state's altitude is 500 exp(-al); its middle sweep's chain
        // gives the start of the sweep up to 500 km
        const double alt = 500.0 * std::exp(-al);
        const double alm = std::log(alt / f1.low_z);
        const int nm = 1 + (int)std::floor(alm / kLnStepMiddle);
        double mz, mzend;
        sweep_chain(f1.low_zend, std::exp(alm / nm), nm, &mz, &mzend);
        const double alu = std::log(500.0 / mz);
        g.n = n_force > 0 ? n_force : 1 + (int)std::floor(alu / kLnStepMiddle);
        g.zr = std::exp(alu / g.n);
        g.zend_start = mzend;
        g.ain_z = mz;
    }
    return g;
}

// The quadrature's Boole sum (boole_sweep's arithmetic), leaving out the
// intervals ex0..ex1.
double sweep_sum_ex(const Geometry& g, const jb::JbFit& f1, Family fam, const double* tc, int ex0, int ex1) {
    using namespace jb;
    double ain = (fam == kMid ? f1.low_gravl : (fam == kUpHigh ? f1.mid_gravl : grav(g.ain_z))) /
                 local_temp(g.ain_z, tc);
    double sum = 0.0, zend = g.zend_start;
    for (int i = 0; i < g.n; ++i) {
        double zz = zend;
        zend = g.zr * zz;
        const double dz = 0.25 * (zend - zz);
        double sum1 = kW0 * ain;
        for (int j = 1; j < 5; ++j) {
            zz += dz;
            ain = grav(zz) / local_temp(zz, tc);
            sum1 += (j == 1 || j == 3 ? kW1 : (j == 2 ? kW2 : kW0)) * ain;
        }
        if (!(i >= ex0 && i <= ex1)) sum += dz * sum1;
    }
    return sum;
}

double family_sum(Family fam, const jb::JbFit& f1, double al, double tinf, int ex0, int ex1) {
    const Temp T = temp_profile(tinf);
    return sweep_sum_ex(geometry(fam, f1, al), f1, fam, T.tc, ex0, ex1);
}

// Intervals whose nodes (carry included) come within kBreakAbove of the
// 125 km break of the temperature profile anywhere in [a, b] (where its form
// changes, the sum has a kink in the altitude): node altitudes grow
// monotonically with the log-ratio inside a segment, so the two ends, with
// the segment's own interval count n, bracket them.
constexpr double kBreakAbove = 1e-6;
void break_intervals(Family fam, const jb::JbFit& f1, double a, double b, int n, int32_t* ex) {
    int lo = 1 << 30, hi = -1;
    for (double al : {a, b}) {
        const Geometry g = geometry(fam, f1, al, n);
        double zend = g.zend_start, zlast = g.zend_start;
        for (int i = 0; i < g.n; ++i) {
            double zz = zend;
            zend = g.zr * zz;
            const double dz = 0.25 * (zend - zz);
            const double first = std::fmin(zlast, zz);
            zz += dz;
            zz += dz;
            zz += dz;
            zz += dz;
            if (first <= 125.0 + kBreakAbove && zz >= 125.0 - 1e-6) {
                lo = std::min(lo, i);
                hi = std::max(hi, i);
            }
            zlast = zz;
        }
    }
    ex[0] = hi >= 0 ? lo : -1;
    ex[1] = hi >= 0 ? hi : -1;
}

bool build_family(Family fam, const jb::JbFit& f1, double tlo, double thi, int nseg, double step, double rlo,
                  double rhi, double (*rng)[2], int32_t (*ex)[2], double* coef, double* worst) {
    typedef long double LD;
    const LD pi = 3.14159265358979323846264338327950288L;
    const int KA = jb::kFit2A, KT = jb::kFit2T;
    double w = 0.0;
    std::vector<double> vals((size_t)KA * KT);
    std::vector<LD> ca((size_t)KA * KA), ct((size_t)KT * KT);  // cos(pi p (k + 1/2) / K)
    for (int p = 0; p < KA; ++p)
        for (int k = 0; k < KA; ++k) ca[(size_t)p * KA + k] = cosl(pi * p * (k + 0.5L) / KA);
    for (int q = 0; q < KT; ++q)
        for (int j = 0; j < KT; ++j) ct[(size_t)q * KT + j] = cosl(pi * q * (j + 0.5L) / KT);
    for (int s = 0; s < nseg; ++s) {
        double* c = coef + (size_t)s * KA * KT;
        const double a = std::fmax(s * step, rlo), b = std::fmin((s + 1) * step, rhi);
        rng[s][0] = a;
        rng[s][1] = b;
        ex[s][0] = ex[s][1] = -1;
        if (!(b > a)) {  // not reachable: an empty series (never used)
            for (int i = 0; i < KA * KT; ++i) c[i] = 0.0;
            rng[s][1] = a + 1.0;
            continue;
        }
        break_intervals(fam, f1, a, b, s + 1, ex[s]);
        for (int k = 0; k < KA; ++k) {
            const double xa = (double)cosl(pi * (k + 0.5L) / KA);
            const double al = 0.5 * (a + b) + 0.5 * (b - a) * xa;
            for (int j = 0; j < KT; ++j) {
                const double xt = (double)cosl(pi * (j + 0.5L) / KT);
                vals[(size_t)k * KT + j] =
                    family_sum(fam, f1, al, 0.5 * (thi + tlo) + 0.5 * (thi - tlo) * xt, ex[s][0], ex[s][1]);
            }
        }
        for (int p = 0; p < KA; ++p)
            for (int q = 0; q < KT; ++q) {
                LD acc = 0.0L;
                for (int k = 0; k < KA; ++k) {
                    LD row = 0.0L;
                    for (int j = 0; j < KT; ++j) row += (LD)vals[(size_t)k * KT + j] * ct[(size_t)q * KT + j];
                    acc += row * ca[(size_t)p * KA + k];
                }
                c[(size_t)p * KT + q] = (double)((p == 0 ? 1.0L : 2.0L) / KA * (q == 0 ? 1.0L : 2.0L) / KT * acc);
            }
        // check off the sampling grid: series + exact intervals = quadrature
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 5; ++j) {
                const double fa = (i + 0.37) / 6.0, ft = (j + 0.61) / 5.0;
                const double al = a + (b - a) * fa, t = tlo + (thi - tlo) * ft;
                const double full = family_sum(fam, f1, al, t, -1, -1);
                const double part = family_sum(fam, f1, al, t, ex[s][0], ex[s][1]);
                const double got = jb::cheb2_eval(c, jb::fit2_x(rng[s], al), (2.0 * t - (thi + tlo)) / (thi - tlo)) +
                                   (full - part);
                // the sums enter the density through exp(-sum M / R*): below a
                // sum of 1 the absolute error is what moves the density
                w = std::fmax(w, std::fabs(got - full) / std::fmax(std::fabs(full), 1.0));
            }
    }
    *worst = w;
    return w <= 1e-13;
}

}  // namespace fit2

// Builds f2 over the exospheric temperatures [tlo, thi]; worst[3] = the
// families' worst relative errors.
void build_jb_fit2(const jb::JbFit& f1, double tlo, double thi, jb::JbFit2& f2, double* worst) {
    using namespace jb;
    f2 = JbFit2{};
    f2.tlo = tlo;
    f2.thi = thi;
    if (!(f1.valid && f2.tlo >= f1.lo && f2.thi <= f1.hi && f2.thi > f2.tlo)) {
        worst[0] = worst[1] = worst[2] = -1.0;
        return;
    }
    const double lmid_lo = std::log(105.0 / f1.low_z), lmid_hi = std::log(500.0 / f1.low_z);
    f2.valid_mid = fit2::build_family(fit2::kMid, f1, f2.tlo, f2.thi, kFit2Mid, kLnStepMiddle, lmid_lo, lmid_hi,
                                      f2.mid_rng, f2.mid_ex, &f2.mid[0][0][0], &worst[0]);
    f2.valid_uplow = fit2::build_family(fit2::kUpLow, f1, f2.tlo, f2.thi, kFit2UpLow, kLnStepMiddle, 1e-9,
                                        std::log(500.0 / 105.0), f2.uplow_rng, f2.uplow_ex, &f2.uplow[0][0][0],
                                        &worst[1]);
    f2.valid_uphigh = fit2::build_family(fit2::kUpHigh, f1, f2.tlo, f2.thi, kFit2UpHigh, kLnStepUpper,
                                         std::log(500.0 / f1.mid_z), std::log(2500.0 / f1.mid_z), f2.uphigh_rng,
                                         f2.uphigh_ex, &f2.uphigh[0][0][0], &worst[2]);
}

bool build_jb_fit(jb::JbFit& f, double* worst) {
    typedef long double LD;
    const int N = jb::kFitTerms;
    f.valid = 0;
    f.terms = N;
    f.lo = 300.0;
    f.hi = 3500.0;
    std::vector<LD> fl(N), fm(N);
    jb::Sweep lo, mid;
    for (int k = 0; k < N; ++k) {
        const LD x = cosl(3.14159265358979323846264338327950288L * (k + 0.5L) / N);
        const double t = 0.5 * (f.hi + f.lo) + 0.5 * (f.hi - f.lo) * (double)x;
        sweep_sums(t, &lo, &mid);
        fl[k] = lo.sum;
        fm[k] = mid.sum;
        if (k == 0) {
            f.low_z = lo.z;
            f.low_zend = lo.zend;
            f.low_mb2 = lo.mb;
            f.low_gravl = lo.gravl;
            f.mid_z = mid.z;
            f.mid_zend = mid.zend;
            f.mid_gravl = mid.gravl;
        } else if (lo.z != f.low_z || lo.zend != f.low_zend || mid.z != f.mid_z || mid.zend != f.mid_zend) {
            return false;  // node altitudes must not depend on T_inf
        }
    }
    for (int j = 0; j < N; ++j) {
        LD sl = 0, sm = 0;
        for (int k = 0; k < N; ++k) {
            const LD c = cosl(3.14159265358979323846264338327950288L * j * (k + 0.5L) / N);
            sl += fl[k] * c;
            sm += fm[k] * c;
        }
        f.low[j] = (double)((j == 0 ? 1.0L : 2.0L) / N * sl);
        f.mid[j] = (double)((j == 0 ? 1.0L : 2.0L) / N * sm);
    }
    double w = 0.0;
    for (int i = 0; i < 257; ++i) {
        const double t = f.lo + (f.hi - f.lo) * (i + 0.5) / 257.0;
        sweep_sums(t, &lo, &mid);
        const double a = jb::cheb_eval(f.low, N, f.lo, f.hi, t);
        const double b = jb::cheb_eval(f.mid, N, f.lo, f.hi, t);
        w = std::max(w, std::max(std::fabs(a - lo.sum) / std::fabs(lo.sum), std::fabs(b - mid.sum) / std::fabs(mid.sum)));
    }
    *worst = w;
    f.valid = w <= 4e-15 ? 1 : 0;
    return f.valid != 0;
}

}  // namespace

struct bqp_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bqp_force_config cfg{};
    Coeffs coeffs;
    int parsed_order = 0;
    double* d_tab = nullptr;
    int ncells = 0;
    size_t tab_bytes = 0;
    int use_smem = 0;
    void* d_tab_split = nullptr;  // split-precision table (cfg.split_degree > 0)
    int split_ls = 0;             // its last FP64 row
    uint32_t split_bytes = 0;
    unsigned long long* d_queue = nullptr;
    void* d_ws = nullptr;
    size_t ws_bytes = 0;
    void* d_pws = nullptr;  // stage-synchronous engine buffers
    size_t pws_bytes = 0;
    jb::JbFit* d_fit = nullptr;  // JB2008 fixed-node sweep fits (device)
    double fit_worst = -1.0;
    jb::JbFit h_fit{};            // host copy of the same
    jb::JbFit2* d_fit2 = nullptr; // altitude-dependent sweep fits over the T_inf range below
    double fit2_tinf[2] = {};     // the range they were built for
    double fit2_worst[3] = {-1.0, -1.0, -1.0};
    bool fit2_built = false;
    SpaceWeather sw;              // space-weather tables (bqp_ctx_set_jb_drivers), host copy
    double sw_span[2] = {};       // UTC span the fits are sized for (0, 0: the whole table)
    double* d_sw_solar = nullptr;
    int32_t* d_sw_dtc = nullptr;
    jb::DriverTable dtab{};       // the device copy as the kernels see it (n_solar 0: none)
    double* d_eph[2] = {nullptr, nullptr};  // Sun / Moon catalogues (bqp_ctx_set_ephemeris)
    EphemTable eph[2] = {};                 // their device views (n 0: the analytic series)
    double sun_rate = kSunRateAnalytic;     // bound of the Sun direction's rate, rad/day
    EclState* d_ecl = nullptr;              // eclipse coordinator state, one per SRP row
    int64_t ecl_cap = 0;
    bool profile = false;  // kernel timing on (bqp_ctx_profile)
    KernelTimes times{};
    Model* sur = nullptr;          // learned gravity surrogate (bqp_surrogate_*)
    double* d_tab_low = nullptr;   // FP64 table of degrees <= BQP_SURROGATE_DEGREE
    uint32_t low_bytes = 0;
    // IAU 2006/2000A Earth-fixed frame (bqp_ctx_set_frame): the segment
    // authority (null: the GMST rotation) and the device copy of the
    // segments of the latest batch
    std::unique_ptr<ft::Authority> frame;
    ft::FrameSeg* d_fseg = nullptr;
    int64_t* d_fkey = nullptr;
    int64_t fseg_cap = 0;
    ft::FrameIntervals* d_fivl = nullptr;
    ft::FrameTab ftab{};
    bool frame_span = false;  // the table covers a span set once (bqp_ctx_set_frame_span)
};

namespace {

int validate_cfg(const bqp_force_config* c) {
    if (!c) return fail(BQP_E_ARG, "null config");
    if (c->order < 0 || c->order > kMaxOrder)
        return fail(BQP_E_ARG, "order must be in 0..%d, got %d", kMaxOrder, c->order);
    if (c->force_flags & BQP_FORCE_SRP) {
        if (c->method == BQP_METHOD_DOPRI5_COMPAT)
            return fail(BQP_E_UNSUPPORTED, "binary-eclipse SRP runs with the dopri5 / dop853 / vern7 / vern9 steppers");
        if (c->error_control != 0)
            return fail(BQP_E_UNSUPPORTED, "binary-eclipse SRP runs with absolute error control (error_control 0)");
    }
    if (!(std::isfinite(c->cr) && c->cr >= 0.0 && std::isfinite(c->p_sun) && c->p_sun >= 0.0))
        return fail(BQP_E_ARG, "cr and p_sun must be finite and >= 0");
    if (c->force_flags & ~(BQP_FORCE_DRAG | BQP_FORCE_SUN | BQP_FORCE_MOON | BQP_FORCE_SRP))
        return fail(BQP_E_ARG, "unknown force flags 0x%x", c->force_flags);
    if ((c->force_flags & BQP_FORCE_DRAG) && (c->atm_model < 4 || c->atm_model > 7))
        return fail(BQP_E_UNSUPPORTED, "atm_model %d is not a JB2008 profile; use 4 (exact) or 5, 6, 7 (coarse)",
                    c->atm_model);
    if (c->method < 0 || c->method > 4) return fail(BQP_E_ARG, "unknown method %d", c->method);
    if (c->error_control == 0) {
        if (!(std::isfinite(c->eps) && c->eps > 0.0)) return fail(BQP_E_ARG, "eps must be finite and > 0");
    } else if (c->error_control == 1) {
        if (c->method == BQP_METHOD_DOPRI5_COMPAT)
            return fail(BQP_E_ARG, "the DOPRI5 compatibility loop has absolute error control only");
        if (!(std::isfinite(c->rtol) && c->rtol > 0.0 && std::isfinite(c->atol) && c->atol >= 0.0))
            return fail(BQP_E_ARG, "rtol must be finite and > 0, atol finite and >= 0");
    } else {
        return fail(BQP_E_ARG, "error_control must be 0 or 1");
    }
    if (!(std::isfinite(c->dt_max) && c->dt_max > 0.0)) return fail(BQP_E_ARG, "dt_max must be finite and > 0");
    if (!(std::isfinite(c->am_ratio) && c->am_ratio >= 0.0 && std::isfinite(c->cd) && c->cd >= 0.0))
        return fail(BQP_E_ARG, "am_ratio and cd must be finite and >= 0");
    if (c->max_steps <= 0 || c->max_attempts <= 0) return fail(BQP_E_ARG, "step budgets must be > 0");
    if (!(c->max_kernel_seconds > 0.0)) return fail(BQP_E_ARG, "max_kernel_seconds must be > 0");
    if (c->engine != BQP_ENGINE_PIPELINE && c->engine != BQP_ENGINE_PERSISTENT)
        return fail(BQP_E_ARG, "unknown engine %d", c->engine);
    if (c->gravity_threads < 0 || c->gravity_threads > 256 || c->gravity_threads % 32)
        return fail(BQP_E_ARG, "gravity_threads must be a multiple of 32 in 0..256");
    if (c->gravity_slots != 0 && c->gravity_slots != 1 && c->gravity_slots != 2 && c->gravity_slots != 4)
        return fail(BQP_E_ARG, "gravity_slots must be 0, 1, 2 or 4");
    if (c->split_degree != 0 && (c->split_degree < 4 || c->split_degree > kMaxOrder))
        return fail(BQP_E_ARG, "split_degree must be 0 (plain FP64) or in 4..%d, got %d", kMaxOrder,
                    c->split_degree);
    if (c->split_degree != 0 && c->engine == BQP_ENGINE_PERSISTENT)
        return fail(BQP_E_UNSUPPORTED, "split precision runs in the stage-synchronous engine");
    if (c->drag_fp32 != 0 && c->drag_fp32 != 1) return fail(BQP_E_ARG, "drag_fp32 must be 0 or 1");
    if (c->drag_fp32 && (c->force_flags & BQP_FORCE_DRAG) && c->atm_model == 4)
        return fail(BQP_E_UNSUPPORTED,
                    "the FP32 JB2008 density is built for the coarse profiles (atm_model 5, 6, 7), not the exact model");
    if (c->surrogate != 0 && c->surrogate != 1) return fail(BQP_E_ARG, "surrogate must be 0 or 1");
    if (c->surrogate && c->engine == BQP_ENGINE_PERSISTENT)
        return fail(BQP_E_UNSUPPORTED, "the surrogate gravity runs in the stage-synchronous engine");
    if (c->surrogate && c->split_degree)
        return fail(BQP_E_ARG, "choose the surrogate or split precision, not both");
    if (!(std::isfinite(c->surrogate_check) && c->surrogate_check >= 0.0))
        return fail(BQP_E_ARG, "surrogate_check must be finite and >= 0");
    if (c->drag_fp32 && c->engine == BQP_ENGINE_PERSISTENT)
        return fail(BQP_E_UNSUPPORTED, "the FP32 density runs in the stage-synchronous engine");
    return 0;
}

ForceParams force_params(const bqp_ctx* ctx) {
    const bqp_force_config& c = ctx->cfg;
    ForceParams fp{};
    fp.order = c.order;
    fp.gravity_on = c.order > 0;
    fp.drag = (c.force_flags & BQP_FORCE_DRAG) ? 1 : 0;
    fp.sun = (c.force_flags & BQP_FORCE_SUN) ? 1 : 0;
    fp.moon = (c.force_flags & BQP_FORCE_MOON) ? 1 : 0;
    fp.ground_check = c.ground_check;
    fp.atm_model = (c.force_flags & BQP_FORCE_DRAG) ? c.atm_model : 4;
    fp.drag_fp32 = c.drag_fp32;
    fp.srp = (c.force_flags & BQP_FORCE_SRP) ? 1 : 0;
    fp.cr = c.cr;
    fp.p_sun = c.p_sun;
    fp.sun_rate = ctx->sun_rate;
    fp.earth_radius = c.earth_radius;
    fp.omega = c.omega_earth;
    fp.mu_sun = c.mu_sun;
    fp.mu_moon = c.mu_moon;
    fp.drivers = {c.jb_drivers[0], c.jb_drivers[1], c.jb_drivers[2], c.jb_drivers[3], c.jb_drivers[4],
                  c.jb_drivers[5], c.jb_drivers[6], c.jb_drivers[7], c.jb_drivers[8]};
    fp.dtab = ctx->dtab;
    fp.eph_sun = ctx->eph[0];
    fp.eph_moon = ctx->eph[1];
    // the sweep fits replace the exact model's quadrature only
    fp.fit = (c.drag_quadrature || !fp.drag || fp.atm_model != 4) ? nullptr : ctx->d_fit;
    fp.fit2 = fp.fit ? ctx->d_fit2 : nullptr;
    fp.frame = ctx->ftab;
    return fp;
}

// The IAU frame's segments for a batch: every segment holding an instant of
// a row's [epoch + min(t0, tf), epoch + max(t0, tf)] (one more on each
// side), built on the host (kept by the authority) and copied to the device
// sorted by key.  Rows whose instants have no segment fail on the device
// with the frame-time status.  Host arrays.
int frame_prepare_host_impl(bqp_ctx* ctx, int64_t n, const double* epoch, const double* lo, const double* hi) {
    if (!ctx->frame) {
        ctx->ftab = ft::FrameTab{};
        return 0;
    }
    if (ctx->frame_span) return 0;
    std::vector<std::pair<int32_t, int64_t>> want;
    const double pad = ft::kSegWidth;
    double tmin = INFINITY, tmax = -INFINITY;
    std::vector<std::pair<double, double>> spans;
    for (int64_t i = 0; i < n; ++i) {
        double tai0;
        if (!ft::tai_seconds_from_utc_jd(epoch[i], &tai0)) continue;
        const double a = tai0 + std::min(lo[i], hi[i]) - pad, b = tai0 + std::max(lo[i], hi[i]) + pad;
        if (!(std::isfinite(a) && std::isfinite(b))) continue;
        spans.push_back({a, b});
        tmin = std::min(tmin, a);
        tmax = std::max(tmax, b);
    }
    // merge overlapping row spans before listing their segments
    std::sort(spans.begin(), spans.end());
    for (size_t i = 0; i < spans.size();) {
        double a = spans[i].first, b = spans[i].second;
        size_t j = i + 1;
        while (j < spans.size() && spans[j].first <= b) b = std::max(b, spans[j++].second);
        ctx->frame->keys_between(a, b, &want);
        i = j;
    }
    std::vector<int64_t> keys;
    std::vector<ft::FrameSeg> segs;
    ctx->frame->ensure(want, &keys, &segs);
    const int64_t m = (int64_t)keys.size();
    cudaError_t e = cudaSuccess;
    if (m > ctx->fseg_cap) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->d_fseg);
        cudaFree(ctx->d_fkey);
        ctx->d_fseg = nullptr;
        ctx->d_fkey = nullptr;
        ctx->fseg_cap = 0;
        const int64_t cap = std::max<int64_t>(m, 64);
        e = cudaMalloc(&ctx->d_fseg, (size_t)cap * sizeof(ft::FrameSeg));
        if (e == cudaSuccess) e = cudaMalloc(&ctx->d_fkey, (size_t)cap * sizeof(int64_t));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(frame segments)");
        ctx->fseg_cap = cap;
    }
    if (!ctx->d_fivl) {
        e = cudaMalloc(&ctx->d_fivl, sizeof(ft::FrameIntervals));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(frame intervals)");
    }
    // synchronous copies: the host vectors go out of scope on return
    if (m > 0) e = cudaMemcpyAsync(ctx->d_fseg, segs.data(), (size_t)m * sizeof(ft::FrameSeg),
                                   cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess && m > 0)
        e = cudaMemcpyAsync(ctx->d_fkey, keys.data(), (size_t)m * sizeof(int64_t), cudaMemcpyHostToDevice,
                            ctx->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ctx->d_fivl, &ctx->frame->intervals(), sizeof(ft::FrameIntervals),
                            cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "frame segment upload");
    ctx->ftab.mode = 1;
    ctx->ftab.nseg = (int32_t)m;
    ctx->ftab.seg = ctx->d_fseg;
    ctx->ftab.key = ctx->d_fkey;
    ctx->ftab.ivl = ctx->d_fivl;
    return 0;
}

// The host side builds with standard containers and threads: a failure to
// allocate comes back as a status, not as an exception through the C ABI.
int frame_prepare_host(bqp_ctx* ctx, int64_t n, const double* epoch, const double* lo, const double* hi) {
    try {
        return frame_prepare_host_impl(ctx, n, epoch, lo, hi);
    } catch (const std::exception& e) {
        return fail(BQP_E_NOMEM, "frame segments: %s", e.what());
    }
}

// The same for device arrays of epochs and end times (start d_t0 per row,
// or the common t0 when it is null).
int frame_prepare_dev(bqp_ctx* ctx, int64_t n, const double* d_epoch, double t0, const double* d_tf,
                      const double* d_t0 = nullptr) {
    if (!ctx->frame) {
        ctx->ftab = ft::FrameTab{};
        return 0;
    }
    if (ctx->frame_span) return 0;  // no readback: the preset span's table stands
    std::vector<double> ep, tf, lo;
    try {
        ep.resize((size_t)n);
        tf.resize((size_t)n);
        lo.assign((size_t)n, t0);
    } catch (const std::exception& ex) {
        return fail(BQP_E_NOMEM, "frame span readback: %s", ex.what());
    }
    cudaError_t e = cudaSuccess;
    if (n > 0 && d_t0) e = cudaMemcpyAsync(lo.data(), d_t0, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && n > 0)
        e = cudaMemcpyAsync(ep.data(), d_epoch, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && n > 0)
        e = cudaMemcpyAsync(tf.data(), d_tf, (size_t)n * 8, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "frame span readback");
    return frame_prepare_host(ctx, n, ep.data(), lo.data(), tf.data());
}

// Builds (once per driver set) the altitude-dependent sweep fits; they are
// used only where the quadrature would otherwise run and the 1-D fits hold.
int ensure_fit2(bqp_ctx* ctx) {
    const bqp_force_config& c = ctx->cfg;
    if (!(c.force_flags & BQP_FORCE_DRAG) || c.drag_quadrature || !ctx->d_fit || c.atm_model != 4) return 0;
    // the fits depend only on the T_inf range the drivers can produce
    double tinf[2] = {0.0, 0.0};
    if (ctx->dtab.n_solar > 0) {
        if (!space_weather_tinf_range(ctx->sw, ctx->sw_span[0], ctx->sw_span[1], &tinf[0], &tinf[1]))
            tinf[0] = tinf[1] = 0.0;  // no usable day: the quadrature runs
    } else {
        const jb::Drivers d{c.jb_drivers[0], c.jb_drivers[1], c.jb_drivers[2], c.jb_drivers[3], c.jb_drivers[4],
                            c.jb_drivers[5], c.jb_drivers[6], c.jb_drivers[7], c.jb_drivers[8]};
        fit2::tinf_range(d, &tinf[0], &tinf[1]);
    }
    if (ctx->fit2_built && ctx->fit2_tinf[0] == tinf[0] && ctx->fit2_tinf[1] == tinf[1]) return 0;
    std::unique_ptr<jb::JbFit2> f2(new jb::JbFit2());
    build_jb_fit2(ctx->h_fit, tinf[0], tinf[1], *f2, ctx->fit2_worst);
    if (!ctx->d_fit2) {
        cudaError_t e = cudaMalloc(&ctx->d_fit2, sizeof(jb::JbFit2));
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(JB2008 sweep fits)");
    }
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaError_t e = cudaMemcpy(ctx->d_fit2, f2.get(), sizeof(jb::JbFit2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "JB2008 sweep fit upload");
    ctx->fit2_tinf[0] = tinf[0];
    ctx->fit2_tinf[1] = tinf[1];
    ctx->fit2_built = true;
    return 0;
}

CtrlParams ctrl_params(const bqp_ctx* ctx) {
    const bqp_force_config& c = ctx->cfg;
    CtrlParams p{};
    p.scaled = c.error_control;
    p.max_rejects = 50;
    p.eps = c.error_control == 0 ? std::max(c.eps, 1e-12) : c.eps;  // integrator.rs:427
    p.rtol = c.rtol;
    p.atol = c.atol;
    p.h_min = 1e-12;
    p.h_max = c.dt_max;
    p.max_steps = c.max_steps;
    p.max_attempts = c.max_attempts;
    p.max_kernel_ns = c.max_kernel_seconds > 0.0 ? (int64_t)(c.max_kernel_seconds * 1e9) : 0;
    return p;
}

int upload_table(bqp_ctx* ctx) {
    std::vector<double> tab = build_gravity_table(ctx->coeffs, ctx->cfg.order);
    ctx->ncells = gravity_cells(ctx->cfg.order);
    ctx->tab_bytes = tab.size() * sizeof(double);
    ctx->use_smem = ctx->tab_bytes <= kSmemLimit ? 1 : 0;
    if (ctx->d_tab) cudaFree(ctx->d_tab);
    ctx->d_tab = nullptr;
    cudaError_t e = cudaMalloc(&ctx->d_tab, ctx->tab_bytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(gravity table)");
    e = cudaMemcpy(ctx->d_tab, tab.data(), ctx->tab_bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(gravity table)");
    // split precision: FP64 cells of rows <= ls, FP32 cells of the rest
    if (ctx->d_tab_split) cudaFree(ctx->d_tab_split);
    ctx->d_tab_split = nullptr;
    ctx->split_ls = 0;
    ctx->split_bytes = 0;
    const int N = ctx->cfg.order, ls = ctx->cfg.split_degree + 1;
    if (ctx->cfg.split_degree > 0 && ls <= N) {
        std::vector<unsigned char> buf(gravity_table_bytes(N, ls));
        double* lo = reinterpret_cast<double*>(buf.data());
        float* hi = reinterpret_cast<float*>(buf.data() + (size_t)split_lo_cells(ls) * kCellDoubles * 8);
        const int last = N + 1;
        for (int j = 0; j <= last; ++j) {
            const size_t col = (size_t)gravity_col_offset(N, j);
            for (int l = j; l <= last; ++l) {
                const double* c = &tab[(col + (l - j)) * kCellDoubles];
                if (j <= ls && l <= ls) {
                    double* o = lo + ((size_t)split_lo_offset(ls, j) + (l - j)) * kCellDoubles;
                    for (int k = 0; k < kCellDoubles; ++k) o[k] = c[k];
                } else {
                    const int first = j <= ls ? ls + 1 : j;  // first FP32 row of column j
                    float* o = hi + ((size_t)split_hi_offset(N, ls, j) + (l - first)) * kCellDoubles;
                    for (int k = 0; k < kCellDoubles; ++k) o[k] = (float)c[k];
                }
            }
        }
        e = cudaMalloc(&ctx->d_tab_split, buf.size());
        if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(split gravity table)");
        e = cudaMemcpy(ctx->d_tab_split, buf.data(), buf.size(), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(split gravity table)");
        ctx->split_ls = ls;
        ctx->split_bytes = (uint32_t)buf.size();
    }
    return 0;
}

int surrogate_stage_args(bqp_ctx* ctx, SurrogateRef& S);  // below, with the surrogate entry points

// The table the gravity kernels read: split precision when configured.
GravTable grav_table(const bqp_ctx* ctx) {
    GravTable T{};
    T.order = ctx->cfg.order;
    if (ctx->split_ls > 0) {
        T.tab = static_cast<const double*>(ctx->d_tab_split);
        T.ls = ctx->split_ls;
        T.bytes = ctx->split_bytes;
    } else {
        T.tab = ctx->d_tab;
        T.ls = 0;
        T.bytes = (uint32_t)ctx->tab_bytes;
    }
    T.in_smem = T.bytes <= kSmemLimit ? 1 : 0;
    return T;
}

// Device workspace carve-out for the host-buffer entry points.  Each entry
// point runs its carve sequence twice: once on a null base to size the
// workspace, then on the allocated base, so the two can never disagree.
struct Carve {
    char* base;
    size_t off = 0;
    template <typename T>
    T* take(size_t count) {
        off = (off + 255) & ~(size_t)255;
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += count * sizeof(T);
        return p;
    }
};

int ensure_ws(bqp_ctx* ctx, size_t bytes) {
    if (bytes <= ctx->ws_bytes) return 0;
    if (ctx->d_ws) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(ctx->d_ws);
        ctx->d_ws = nullptr;
        ctx->ws_bytes = 0;
    }
    size_t want = std::max(bytes, (size_t)1 << 20);
    cudaError_t e = cudaMalloc(&ctx->d_ws, want);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(workspace)");
    ctx->ws_bytes = want;
    return 0;
}

int set_device(const bqp_ctx* ctx) {
    cudaError_t e = cudaSetDevice(ctx->device);
    return e == cudaSuccess ? 0 : cuda_fail(e, "cudaSetDevice");
}

int launch_prop(bqp_ctx* ctx, int64_t n, const double* in, int32_t input_equ, const double* epoch,
                double t0, const double* tf, const double* ballistic, int32_t n_t, const double* t_eval,
                int32_t out_mode, double* out, int32_t* status, int64_t* steps, int64_t* evals) {
    PropArgs A{};
    A.n = n;
    A.in = in;
    A.input_equinoctial = input_equ;
    A.epoch = epoch;
    A.t0 = t0;
    A.tf = tf;
    A.ballistic = ballistic;
    A.am0 = ctx->cfg.am_ratio;
    A.cd0 = ctx->cfg.cd;
    A.t_eval = t_eval;
    A.n_t = n_t;
    A.out_mode = out_mode;
    A.out = out;
    A.status = status;
    A.steps = steps;
    A.evals = evals;
    A.queue = ctx->d_queue;
    A.gtab = ctx->d_tab;
    A.ncells = ctx->ncells;
    A.use_smem = ctx->use_smem;
    if (int rc = ensure_fit2(ctx)) return rc;
    if (int rc = frame_prepare_dev(ctx, n, epoch, t0, tf)) return rc;
    A.force = force_params(ctx);
    A.fit_host = A.force.fit ? &ctx->h_fit : nullptr;
    A.ctrl = ctrl_params(ctx);
    A.grav = grav_table(ctx);
    if (ctx->cfg.surrogate) {
        if (int rc = surrogate_stage_args(ctx, A.sur)) return rc;
    }
    if (A.force.srp) {
        if (n > ctx->ecl_cap) {
            if (ctx->d_ecl) {
                cudaStreamSynchronize(ctx->stream);
                cudaFree(ctx->d_ecl);
                ctx->d_ecl = nullptr;
                ctx->ecl_cap = 0;
            }
            cudaError_t e = cudaMalloc(&ctx->d_ecl, (size_t)n * sizeof(EclState));
            if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(eclipse coordinator state)");
            ctx->ecl_cap = n;
        }
        A.ecl = ctx->d_ecl;
    }
    if (ctx->cfg.engine == BQP_ENGINE_PIPELINE) {
        const size_t need = pipeline_bytes(n);
        if (need > ctx->pws_bytes) {
            if (ctx->d_pws) {
                cudaStreamSynchronize(ctx->stream);
                cudaFree(ctx->d_pws);
                ctx->d_pws = nullptr;
                ctx->pws_bytes = 0;
            }
            cudaError_t e = cudaMalloc(&ctx->d_pws, need);
            if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(pipeline buffers)");
            ctx->pws_bytes = need;
        }
        PipeBufs P{};
        pipeline_carve(P, ctx->d_pws, n);
        P.iau = A.force.frame.mode == 1 ? 1 : 0;
        cudaError_t e = launch_pipeline(A, P, ctx->cfg.method, ctx->stream, ctx->cfg.max_kernel_seconds,
                                        ctx->cfg.gravity_threads, ctx->cfg.gravity_slots,
                                        ctx->profile ? &ctx->times : nullptr);
        if (e != cudaSuccess) return cuda_fail(e, "pipeline");
        return 0;
    }
    cudaError_t e = cudaMemsetAsync(ctx->d_queue, 0, sizeof(unsigned long long), ctx->stream);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(queue)");
    cudaEvent_t ev[2] = {nullptr, nullptr};
    if (ctx->profile) {
        cudaEventCreate(&ev[0]);
        cudaEventCreate(&ev[1]);
        cudaEventRecord(ev[0], ctx->stream);
    }
    e = launch_propagate(A, ctx->cfg.method, 256, 0, ctx->stream);
    if (ctx->profile) {
        cudaEventRecord(ev[1], ctx->stream);
        float ms = 0.0f;
        if (e == cudaSuccess && cudaEventSynchronize(ev[1]) == cudaSuccess &&
            cudaEventElapsedTime(&ms, ev[0], ev[1]) == cudaSuccess) {
            ctx->times.ms[kKcPersistent] += ms;
            ctx->times.launches[kKcPersistent] += 1;
        }
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
    }
    if (e != cudaSuccess) return cuda_fail(e, "k_propagate launch");
    return 0;
}

int check_prop_args(int64_t n, const double* in, const double* epoch, double t0, const double* tf,
                    const double* out, const int32_t* status) {
    if (n < 0) return fail(BQP_E_ARG, "n must be >= 0");
    if (n > 0 && (!in || !epoch || !tf || !out || !status))
        return fail(BQP_E_ARG, "null buffer");
    if (!std::isfinite(t0)) return fail(BQP_E_ARG, "t0 must be finite");
    return 0;
}

int check_grid(int32_t n_t, const double* t_eval) {
    if (n_t <= 0 || !t_eval) return fail(BQP_E_ARG, "t_eval must be a non-empty array");
    for (int32_t i = 0; i < n_t; ++i) {
        if (!std::isfinite(t_eval[i])) return fail(BQP_E_ARG, "t_eval[%d] is not finite", i);
        if (i > 0 && !(t_eval[i] > t_eval[i - 1]))
            return fail(BQP_E_ARG, "t_eval must be strictly increasing (index %d)", i);
    }
    return 0;
}

// --- Keplerian elements (Python kep_to_eci / eci_to_kep, lib.rs:200-221)
void kep2eci(const double* kep, double* out) {
    const double a = kep[0], e = kep[1];
    if (!(a > 0.0) || !(e >= 0.0 && e < 1.0)) {
        for (int i = 0; i < 6; ++i) out[i] = NAN;
        return;
    }
    const double d2r = kPi / 180.0;
    const double inc = kep[2] * d2r, raan = kep[3] * d2r, argp = kep[4] * d2r, nu = kep[5] * d2r;
    const double p = a * (1.0 - e * e);
    const double cn = std::cos(nu), sn = std::sin(nu);
    const double r = p / (1.0 + e * cn);
    const double sp = std::sqrt(kMu / p);
    const double xp = r * cn, yp = r * sn;
    const double vxp = -sp * sn, vyp = sp * (e + cn);
    const double cO = std::cos(raan), sO = std::sin(raan), cw = std::cos(argp), sw = std::sin(argp);
    const double ci = std::cos(inc), si = std::sin(inc);
    const double r00 = cO * cw - sO * sw * ci, r01 = -cO * sw - sO * cw * ci;
    const double r10 = sO * cw + cO * sw * ci, r11 = -sO * sw + cO * cw * ci;
    const double r20 = sw * si, r21 = cw * si;
    out[0] = r00 * xp + r01 * yp;
    out[1] = r10 * xp + r11 * yp;
    out[2] = r20 * xp + r21 * yp;
    out[3] = r00 * vxp + r01 * vyp;
    out[4] = r10 * vxp + r11 * vyp;
    out[5] = r20 * vxp + r21 * vyp;
}

double wrap360(double deg) {
    double x = std::fmod(deg, 360.0);
    if (x < 0.0) x += 360.0;
    return x >= 360.0 ? x - 360.0 : x;
}

void eci2kep(const double* s, double* out) {
    const double r[3] = {s[0], s[1], s[2]}, v[3] = {s[3], s[4], s[5]};
    const double rn = std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    const double v2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    const double rv = r[0] * v[0] + r[1] * v[1] + r[2] * v[2];
    const double energy = 0.5 * v2 - kMu / rn;
    if (!(energy < -1e-12) || !(rn > 0.0)) {
        for (int i = 0; i < 6; ++i) out[i] = NAN;
        return;
    }
    const double h[3] = {r[1] * v[2] - r[2] * v[1], r[2] * v[0] - r[0] * v[2], r[0] * v[1] - r[1] * v[0]};
    const double hn = std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
    const double nvec[2] = {-h[1], h[0]};
    const double nn = std::sqrt(nvec[0] * nvec[0] + nvec[1] * nvec[1]);
    double ev[3];
    for (int i = 0; i < 3; ++i) ev[i] = ((v2 - kMu / rn) * r[i] - rv * v[i]) / kMu;
    const double e = std::sqrt(ev[0] * ev[0] + ev[1] * ev[1] + ev[2] * ev[2]);
    const double a = -kMu / (2.0 * energy);
    const double r2d = 180.0 / kPi;
    const double inc = std::acos(std::max(-1.0, std::min(1.0, h[2] / hn)));
    const bool equatorial = nn < 1e-11 * hn;
    const bool circular = e < 1e-11;
    double raan = equatorial ? 0.0 : std::atan2(nvec[1], nvec[0]);
    double argp = 0.0, nu = 0.0;
    if (!circular) {
        if (!equatorial) {
            argp = std::acos(std::max(-1.0, std::min(1.0, (nvec[0] * ev[0] + nvec[1] * ev[1]) / (nn * e))));
            if (ev[2] < 0.0) argp = 2.0 * kPi - argp;
        } else {
            argp = std::atan2(ev[1], ev[0]);
            if (h[2] < 0.0) argp = -argp;
        }
        nu = std::acos(std::max(-1.0, std::min(1.0, (ev[0] * r[0] + ev[1] * r[1] + ev[2] * r[2]) / (e * rn))));
        if (rv < 0.0) nu = 2.0 * kPi - nu;
    } else if (!equatorial) {
        nu = std::acos(std::max(-1.0, std::min(1.0, (nvec[0] * r[0] + nvec[1] * r[1]) / (nn * rn))));
        if (r[2] < 0.0) nu = 2.0 * kPi - nu;
    } else {
        nu = std::atan2(r[1], r[0]);
        if (h[2] < 0.0) nu = -nu;
    }
    out[0] = a;
    out[1] = e;
    out[2] = inc * r2d;
    out[3] = wrap360(raan * r2d);
    out[4] = wrap360(argp * r2d);
    out[5] = wrap360(nu * r2d);
}

// Sigma-point sets (sigma.cu).  Julier's n + 2 recursion at W0 = 0 with the
// centre dropped (dust_ukf_rs/src/lib.rs:155-200): offsets xi[7][6] such
// that x_i = mean + chol(P) xi_i; weights 1/7.  Merwe scaled set: the
// covariance is scaled by n + lambda before the factorisation.
struct SigmaSet {
    int points = 0;
    double scale = 1.0;  // covariance factor before Cholesky
    double offsets[7 * 6] = {};
    double wm[13] = {}, wc[13] = {};
};

int sigma_set(int32_t set, double alpha, double beta, double kappa, SigmaSet& S) {
    const double n = 6.0;
    if (set == BQP_SIGMA_JULIER7) {
        const double w1 = 1.0 / (n + 1.0);
        double seq[8][6] = {};
        seq[1][0] = -1.0 / std::sqrt(2.0 * w1);
        seq[2][0] = 1.0 / std::sqrt(2.0 * w1);
        double jf = 1.0;
        for (int j = 2; j <= 6; ++j) {
            jf += 1.0;
            const double step = 1.0 / std::sqrt(jf * (jf + 1.0) * w1);
            for (int p = 1; p <= j; ++p) seq[p][j - 1] = -step;
            for (int k = 0; k < 6; ++k) seq[j + 1][k] = 0.0;
            seq[j + 1][j - 1] = jf * step;
        }
        S.points = 7;
        S.scale = 1.0;
        for (int p = 0; p < 7; ++p)
            for (int k = 0; k < 6; ++k) S.offsets[p * 6 + k] = seq[p + 1][k];
        for (int p = 0; p < 7; ++p) S.wm[p] = S.wc[p] = w1;
        return 0;
    }
    if (set == BQP_SIGMA_MERWE13) {
        if (!(std::isfinite(alpha) && alpha > 0.0 && std::isfinite(beta) && std::isfinite(kappa)))
            return fail(BQP_E_ARG, "Merwe sigma set: alpha must be finite and > 0, beta and kappa finite");
        const double lambda = alpha * alpha * (n + kappa) - n;
        const double c = n + lambda;
        if (!(c > 0.0)) return fail(BQP_E_ARG, "Merwe sigma set: n + lambda must be > 0");
        S.points = 13;
        S.scale = c;
        S.wm[0] = lambda / c;
        S.wc[0] = lambda / c + (1.0 - alpha * alpha + beta);
        for (int p = 1; p < 13; ++p) S.wm[p] = S.wc[p] = 1.0 / (2.0 * c);
        return 0;
    }
    return fail(BQP_E_ARG, "unknown sigma set %d", set);
}

}  // namespace

// ======================================================================
extern "C" {

void bqp_force_config_default(bqp_force_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->order = 5;                      // Python kwarg default (lib.rs:240)
    c->force_flags = BQP_FORCE_DRAG | BQP_FORCE_SUN | BQP_FORCE_MOON;
    c->atm_model = 7;
    c->method = BQP_METHOD_DOP853;
    c->error_control = 0;
    c->ground_check = 0;
    c->eps = 1e-8;                     // ForceConfig::default (types.rs:497)
    c->rtol = 1e-10;
    c->atol = 1e-9;
    c->dt_max = 300.0;                 // Python dt_max_s default
    c->am_ratio = 0.01;
    c->cd = 2.2;
    c->earth_radius = kReWgs84;
    c->omega_earth = kEarthOmega;
    c->mu_sun = 1.32712440018e11;      // DE431 (types.rs:461-462)
    c->mu_moon = 4902.800066;
    for (int i = 0; i < 8; ++i) c->jb_drivers[i] = 150.0;
    c->jb_drivers[8] = 0.0;
    c->max_steps = 500000;             // MAX_STEPS (integrator.rs:185)
    c->max_attempts = (int64_t)1 << 40;
    c->max_kernel_seconds = 600.0;
    c->engine = BQP_ENGINE_PIPELINE;
    c->gravity_threads = 256;
    c->gravity_slots = 4;
    c->split_degree = 0;
    c->drag_fp32 = 0;
    c->surrogate = 0;
    c->surrogate_check = 0.0;
    c->cr = 1.3;                       // Python cr default (lib.rs:241)
    c->p_sun = kPSun;                  // ForceConfig::default (types.rs:459)
}

const char* bqp_last_error(void) { return g_err.c_str(); }

int bqp_ctx_create(const char* text, int64_t len, const bqp_force_config* cfg, bqp_ctx** out) {
    if (!out) return fail(BQP_E_ARG, "null out");
    *out = nullptr;
    if (!text || len < 0) return fail(BQP_E_ARG, "null coefficient text");
    int rc = validate_cfg(cfg);
    if (rc) return rc;
    bqp_ctx* ctx = new bqp_ctx();
    ctx->cfg = *cfg;
    std::string why;
    if (!parse_coeffs(text, len, cfg->order, ctx->coeffs, why)) {
        delete ctx;
        return fail(BQP_E_COEFF, "gravity coefficients failed to load: %s", why.c_str());
    }
    ctx->parsed_order = cfg->order;
    cudaError_t e = cudaGetDevice(&ctx->device);
    if (e != cudaSuccess) {
        delete ctx;
        return cuda_fail(e, "cudaGetDevice");
    }
    rc = upload_table(ctx);
    if (!rc) {
        e = cudaMalloc(&ctx->d_queue, sizeof(unsigned long long));
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaMalloc(queue)");
    }
    if (!rc) {
        jb::JbFit& fit = ctx->h_fit;
        if (build_jb_fit(fit, &ctx->fit_worst)) {
            e = cudaMalloc(&ctx->d_fit, sizeof fit);
            if (e == cudaSuccess) e = cudaMemcpy(ctx->d_fit, &fit, sizeof fit, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) rc = cuda_fail(e, "JB2008 fit upload");
        }
    }
    // the drag sweep fits are built here, where allocating is allowed, so the
    // allocation-free entry point finds them current
    if (!rc) rc = ensure_fit2(ctx);
    if (rc) {
        bqp_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    g_err.clear();
    return 0;
}

int bqp_ctx_destroy(bqp_ctx* ctx) {
    if (!ctx) return 0;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    else cudaDeviceSynchronize();
    if (ctx->d_tab) cudaFree(ctx->d_tab);
    if (ctx->d_queue) cudaFree(ctx->d_queue);
    if (ctx->d_ecl) cudaFree(ctx->d_ecl);
    if (ctx->d_ws) cudaFree(ctx->d_ws);
    if (ctx->d_pws) cudaFree(ctx->d_pws);
    if (ctx->d_fit) cudaFree(ctx->d_fit);
    if (ctx->d_tab_split) cudaFree(ctx->d_tab_split);
    if (ctx->d_fit2) cudaFree(ctx->d_fit2);
    if (ctx->d_tab_low) cudaFree(ctx->d_tab_low);
    if (ctx->d_sw_solar) cudaFree(ctx->d_sw_solar);
    if (ctx->d_sw_dtc) cudaFree(ctx->d_sw_dtc);
    for (double* p : ctx->d_eph)
        if (p) cudaFree(p);
    if (ctx->d_fseg) cudaFree(ctx->d_fseg);
    if (ctx->d_fkey) cudaFree(ctx->d_fkey);
    if (ctx->d_fivl) cudaFree(ctx->d_fivl);
    delete ctx->sur;
    delete ctx;
    return 0;
}

int bqp_ctx_set_stream(bqp_ctx* ctx, void* stream) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    ctx->stream = (cudaStream_t)stream;
    return 0;
}

int bqp_ctx_info(const bqp_ctx* ctx, int64_t* info) {
    if (!ctx || !info) return fail(BQP_E_ARG, "null argument");
    info[0] = ctx->cfg.order;
    info[1] = ctx->ncells;
    info[2] = (int64_t)ctx->tab_bytes;
    info[3] = ctx->use_smem;
    return 0;
}

int bqp_ctx_info_fit(const bqp_ctx* ctx, double* worst_rel) {
    if (!ctx || !worst_rel) return fail(BQP_E_ARG, "null argument");
    *worst_rel = ctx->d_fit ? ctx->fit_worst : -1.0;
    return 0;
}

int bqp_jb_fit_check(const double* drivers, double* worst) {
    if (!drivers || !worst) return fail(BQP_E_ARG, "null argument");
    jb::JbFit f1;
    std::unique_ptr<jb::JbFit2> f2(new jb::JbFit2());
    build_jb_fit(f1, &worst[0]);
    const jb::Drivers d{drivers[0], drivers[1], drivers[2], drivers[3], drivers[4],
                        drivers[5], drivers[6], drivers[7], drivers[8]};
    double tlo, thi;
    fit2::tinf_range(d, &tlo, &thi);
    build_jb_fit2(f1, tlo, thi, *f2, worst + 1);
    worst[4] = f2->tlo;
    worst[5] = f2->thi;
    return 0;
}

int bqp_jb_density(int32_t model, int32_t fp32, int64_t n, const double* in, double* out) {
    if (model < 4 || model > 7) return fail(BQP_E_ARG, "model must be 4, 5, 6 or 7, got %d", model);
    if (fp32 && model == 4) return fail(BQP_E_UNSUPPORTED, "the FP32 density is built for models 5, 6, 7");
    if (n < 0 || (n > 0 && (!in || !out))) return fail(BQP_E_ARG, "bad buffers");
    for (int64_t i = 0; i < n; ++i) {
        const double* x = in + 14 * i;
        const jb::Drivers d{x[5], x[6], x[7], x[8], x[9], x[10], x[11], x[12], x[13]};
        out[i] = fp32 ? jb::density_coarse_r<float>(x[0], x[1], x[2], x[3], x[4], d, model)
                      : jb::density_model(x[0], x[1], x[2], x[3], x[4], d, model);
    }
    return 0;
}

int bqp_ecl_scan_check(bqp_ctx* ctx, int64_t n, const double* paths, int32_t warp, double* out) {
    if (!ctx || n < 0 || (n > 0 && (!paths || !out))) return fail(BQP_E_ARG, "bad arguments");
    if (n == 0) return 0;
    if (int rc = set_device(ctx)) return rc;
    double *d_in = nullptr, *d_out = nullptr;
    cudaError_t e = cudaMalloc(&d_in, (size_t)n * 16 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_out, (size_t)n * 7 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_in, paths, (size_t)n * 16 * sizeof(double), cudaMemcpyHostToDevice,
                                              ctx->stream);
    if (e == cudaSuccess) e = launch_ecl_scan(force_params(ctx), n, d_in, d_out, warp, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, (size_t)n * 7 * sizeof(double), cudaMemcpyDeviceToHost,
                                              ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_in);
    cudaFree(d_out);
    return e == cudaSuccess ? 0 : cuda_fail(e, "eclipse scan check");
}

int bqp_ctx_set_jb_drivers(bqp_ctx* ctx, const char* solfsmy, int64_t solfsmy_len, const char* dtcfile,
                           int64_t dtcfile_len, double jd_lo, double jd_hi) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    if (!std::isfinite(jd_lo) || !std::isfinite(jd_hi) || jd_hi < jd_lo)
        return fail(BQP_E_ARG, "span must be finite with jd_lo <= jd_hi");
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    else cudaDeviceSynchronize();
    auto drop = [&] {
        if (ctx->d_sw_solar) cudaFree(ctx->d_sw_solar);
        if (ctx->d_sw_dtc) cudaFree(ctx->d_sw_dtc);
        ctx->d_sw_solar = nullptr;
        ctx->d_sw_dtc = nullptr;
        ctx->dtab = jb::DriverTable{};
        ctx->sw = SpaceWeather{};
        ctx->fit2_built = false;
    };
    if (!solfsmy && !dtcfile) {
        drop();
        return ensure_fit2(ctx);
    }
    SpaceWeather sw;
    const std::string why = parse_space_weather(solfsmy, solfsmy_len, dtcfile, dtcfile_len, &sw);
    if (!why.empty()) return fail(BQP_E_ARG, "space-weather file rejected: %s", why.c_str());
    drop();
    cudaError_t e = cudaMalloc(&ctx->d_sw_solar, sw.solar.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&ctx->d_sw_dtc, sw.dtc.size() * sizeof(int32_t));
    if (e == cudaSuccess)
        e = cudaMemcpy(ctx->d_sw_solar, sw.solar.data(), sw.solar.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(ctx->d_sw_dtc, sw.dtc.data(), sw.dtc.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        drop();
        return cuda_fail(e, "space-weather table upload");
    }
    ctx->sw = std::move(sw);
    ctx->sw_span[0] = jd_lo;
    ctx->sw_span[1] = jd_hi;
    ctx->dtab = {ctx->d_sw_solar, ctx->d_sw_dtc, ctx->sw.first_jd, ctx->sw.n_solar, ctx->sw.n_dtc, ctx->sw.dtc_first};
    return ensure_fit2(ctx);
}

int bqp_ctx_jb_lookup(bqp_ctx* ctx, const double* utc_jd, int64_t n, double* out, int32_t* ok) {
    if (!ctx || (n > 0 && (!utc_jd || !out || !ok))) return fail(BQP_E_ARG, "null argument");
    if (ctx->dtab.n_solar <= 0) return fail(BQP_E_ARG, "no space-weather tables set (bqp_ctx_set_jb_drivers)");
    if (n <= 0) return 0;
    cudaSetDevice(ctx->device);
    double *d_jd = nullptr, *d_out = nullptr;
    int32_t* d_ok = nullptr;
    cudaError_t e = cudaMalloc(&d_jd, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_out, n * 9 * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_ok, n * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_jd, utc_jd, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = launch_jb_lookup(ctx->dtab, d_jd, n, d_out, d_ok, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, n * 9 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ok, d_ok, n * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_jd);
    cudaFree(d_out);
    cudaFree(d_ok);
    if (e != cudaSuccess) return cuda_fail(e, "space-weather lookup");
    return 0;
}

int bqp_ctx_set_frame(bqp_ctx* ctx, int32_t mode, const double* eop, int32_t first_mjd, int32_t n_records) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    if (mode != BQP_FRAME_GMST && mode != BQP_FRAME_IAU2006)
        return fail(BQP_E_ARG, "frame mode must be BQP_FRAME_GMST (0) or BQP_FRAME_IAU2006 (1), got %d", mode);
    if (n_records < 0 || (n_records > 0 && !eop)) return fail(BQP_E_ARG, "bad EOP records");
    if (mode == BQP_FRAME_GMST) {
        if (n_records > 0) return fail(BQP_E_ARG, "EOP records are for the IAU frame");
        ctx->frame.reset();
        ctx->ftab = ft::FrameTab{};
        ctx->frame_span = false;
        return 0;
    }
    if (n_records > 0) {
        if (first_mjd < ft::kOriginMjd - 3)
            return fail(BQP_E_ARG, "EOP records start at MJD %d, before the frame's origin MJD %d", first_mjd,
                        ft::kOriginMjd);
        for (int64_t i = 0; i < (int64_t)n_records * 5; ++i)
            if (!std::isfinite(eop[i])) return fail(BQP_E_ARG, "EOP record %lld is not finite", (long long)(i / 5));
    }
    try {
        ft::Eop e;
        if (n_records > 0) {
            e.first_mjd = first_mjd;
            e.rec.assign(eop, eop + (size_t)n_records * 5);
        }
        ctx->frame.reset(new ft::Authority(e));
    } catch (const std::exception& ex) {
        return fail(BQP_E_NOMEM, "frame authority: %s", ex.what());
    }
    ctx->ftab = ft::FrameTab{};
    ctx->frame_span = false;
    return 0;
}

int bqp_ctx_set_frame_span(bqp_ctx* ctx, double utc_jd_lo, double utc_jd_hi) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    if (!ctx->frame) return fail(BQP_E_ARG, "no IAU frame set (bqp_ctx_set_frame)");
    ctx->frame_span = false;
    if (utc_jd_lo == 0.0 && utc_jd_hi == 0.0) return 0;
    if (!(std::isfinite(utc_jd_lo) && std::isfinite(utc_jd_hi) && utc_jd_hi >= utc_jd_lo))
        return fail(BQP_E_ARG, "bad UTC span");
    int rc = set_device(ctx);
    if (rc) return rc;
    const double ep = utc_jd_lo, lo = 0.0, hi = (utc_jd_hi - utc_jd_lo) * 86400.0 + 2.0;
    if ((rc = frame_prepare_host(ctx, 1, &ep, &lo, &hi))) return rc;
    ctx->frame_span = true;
    return 0;
}

int bqp_ctx_set_ephemeris(bqp_ctx* ctx, int32_t body, const uint8_t* bytes, int64_t len) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    if (body != BQP_BODY_SUN && body != BQP_BODY_MOON) return fail(BQP_E_ARG, "body must be 0 (Sun) or 1 (Moon)");
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    else cudaDeviceSynchronize();
    Ephemeris e;
    if (bytes) {
        const std::string why = parse_ephemeris(bytes, len, body, &e);
        if (!why.empty()) return fail(BQP_E_ARG, "ephemeris catalogue rejected: %s", why.c_str());
    }
    if (ctx->d_eph[body]) cudaFree(ctx->d_eph[body]);
    ctx->d_eph[body] = nullptr;
    ctx->eph[body] = EphemTable{};
    if (body == BQP_BODY_SUN) ctx->sun_rate = bytes ? ephemeris_direction_rate(e) : kSunRateAnalytic;
    if (!bytes) return 0;
    cudaError_t err = cudaMalloc(&ctx->d_eph[body], e.pos.size() * sizeof(double));
    if (err == cudaSuccess)
        err = cudaMemcpy(ctx->d_eph[body], e.pos.data(), e.pos.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (err != cudaSuccess) {
        if (ctx->d_eph[body]) cudaFree(ctx->d_eph[body]);
        ctx->d_eph[body] = nullptr;
        return cuda_fail(err, "ephemeris catalogue upload");
    }
    ctx->eph[body] = e.host_view();
    ctx->eph[body].pos = ctx->d_eph[body];
    return 0;
}

int bqp_ctx_body_positions(bqp_ctx* ctx, int32_t body, const double* utc_jd, int64_t n, double* out) {
    if (!ctx || (n > 0 && (!utc_jd || !out))) return fail(BQP_E_ARG, "null argument");
    if (body != BQP_BODY_SUN && body != BQP_BODY_MOON) return fail(BQP_E_ARG, "body must be 0 (Sun) or 1 (Moon)");
    if (n <= 0) return 0;
    cudaSetDevice(ctx->device);
    double *d_jd = nullptr, *d_out = nullptr;
    cudaError_t e = cudaMalloc(&d_jd, n * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&d_out, n * 3 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_jd, utc_jd, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess) e = launch_body_positions(ctx->eph[body], body, d_jd, n, d_out, ctx->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, n * 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(d_jd);
    cudaFree(d_out);
    if (e != cudaSuccess) return cuda_fail(e, "body positions");
    return 0;
}

int bqp_ephemeris_check(int32_t body, const uint8_t* bytes, int64_t len, const double* utc_jd, int64_t n,
                        double* out, int64_t* n_samples) {
    if (!n_samples || (n > 0 && (!utc_jd || !out))) return fail(BQP_E_ARG, "null argument");
    if (body != BQP_BODY_SUN && body != BQP_BODY_MOON) return fail(BQP_E_ARG, "body must be 0 (Sun) or 1 (Moon)");
    Ephemeris e;
    const std::string why = parse_ephemeris(bytes, len, body, &e);
    if (!why.empty()) return fail(BQP_E_ARG, "ephemeris catalogue rejected: %s", why.c_str());
    *n_samples = e.n;
    const EphemTable T = e.host_view();
    for (int64_t i = 0; i < n; ++i) ephem_position(T, utc_jd[i], out + 3 * i);
    return 0;
}

int bqp_jb_drivers_check(const char* solfsmy, int64_t solfsmy_len, const char* dtcfile, int64_t dtcfile_len,
                         const double* utc_jd, int64_t n, double* out, int32_t* ok, int64_t* counts2) {
    if (!counts2 || (n > 0 && (!utc_jd || !out || !ok))) return fail(BQP_E_ARG, "null argument");
    SpaceWeather sw;
    const std::string why = parse_space_weather(solfsmy, solfsmy_len, dtcfile, dtcfile_len, &sw);
    if (!why.empty()) return fail(BQP_E_ARG, "space-weather file rejected: %s", why.c_str());
    counts2[0] = sw.n_solar;
    counts2[1] = sw.n_dtc;
    const jb::DriverTable T = sw.host_view();
    for (int64_t i = 0; i < n; ++i) {
        jb::Drivers d;
        const bool found = jb::lookup_drivers(T, utc_jd[i], &d);
        const double v[9] = {d.f10, d.f10b, d.s10, d.s10b, d.m10, d.m10b, d.y10, d.y10b, d.dtc};
        for (int k = 0; k < 9; ++k) out[9 * i + k] = found ? v[k] : NAN;
        ok[i] = found ? 1 : 0;
    }
    return 0;
}

int bqp_ctx_profile(bqp_ctx* ctx, int32_t on) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    ctx->profile = on != 0;
    if (ctx->profile) ctx->times = KernelTimes{};
    return 0;
}

int bqp_ctx_profile_read(const bqp_ctx* ctx, double* ms, int64_t* launches) {
    if (!ctx || !ms || !launches) return fail(BQP_E_ARG, "null argument");
    for (int i = 0; i < kKcCount; ++i) {
        ms[i] = ctx->times.ms[i];
        launches[i] = ctx->times.launches[i];
    }
    return 0;
}

int bqp_ctx_set_config(bqp_ctx* ctx, const bqp_force_config* cfg) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    int rc = validate_cfg(cfg);
    if (rc) return rc;
    if (cfg->order > ctx->parsed_order)
        return fail(BQP_E_ARG, "order %d exceeds the parsed field order %d", cfg->order, ctx->parsed_order);
    if ((rc = set_device(ctx))) return rc;
    const int old = ctx->cfg.order, old_split = ctx->cfg.split_degree;
    ctx->cfg = *cfg;
    if (cfg->order != old || cfg->split_degree != old_split) {
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
        if ((rc = upload_table(ctx))) return rc;
    }
    return ensure_fit2(ctx);
}

int bqp_gravity_eval_device(bqp_ctx* ctx, int64_t n, const double* pos, double* acc, int32_t* status) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    if (n < 0 || (n > 0 && (!pos || !acc))) return fail(BQP_E_ARG, "bad buffers");
    int rc = set_device(ctx);
    if (rc) return rc;
    cudaError_t e = launch_gravity(grav_table(ctx), n, pos, acc, status, ctx->stream, ctx->cfg.gravity_threads,
                                   ctx->cfg.gravity_slots);
    return e == cudaSuccess ? 0 : cuda_fail(e, "k_gravity launch");
}

int bqp_gravity_eval(bqp_ctx* ctx, int64_t n, const double* pos, double* acc, int32_t* status) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    if (n < 0 || (n > 0 && (!pos || !acc))) return fail(BQP_E_ARG, "bad buffers");
    if (n == 0) return 0;
    int rc = set_device(ctx);
    if (rc) return rc;
    const size_t b3 = (size_t)n * 3 * sizeof(double);
    double *dp = nullptr, *da = nullptr;
    int32_t* ds = nullptr;
    for (int pass = 0; pass < 2; ++pass) {
        Carve cv{pass ? (char*)ctx->d_ws : nullptr};
        dp = cv.take<double>((size_t)n * 3);
        da = cv.take<double>((size_t)n * 3);
        ds = cv.take<int32_t>((size_t)n);
        if (!pass && (rc = ensure_ws(ctx, cv.off))) return rc;
    }
    cudaError_t e = cudaMemcpyAsync(dp, pos, b3, cudaMemcpyHostToDevice, ctx->stream);
    if (e == cudaSuccess)
        e = launch_gravity(grav_table(ctx), n, dp, da, ds, ctx->stream, ctx->cfg.gravity_threads,
                           ctx->cfg.gravity_slots);
    if (e == cudaSuccess) e = cudaMemcpyAsync(acc, da, b3, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess && status)
        e = cudaMemcpyAsync(status, ds, (size_t)n * 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return e == cudaSuccess ? 0 : cuda_fail(e, "bqp_gravity_eval");
}

int bqp_rhs_eval_device(bqp_ctx* ctx, int64_t n, const double* equ, const double* seg_t0,
                        const double* epoch_jd, const double* t, const double* delta,
                        const double* ballistic, double* out) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    if (n < 0 || (n > 0 && (!equ || !seg_t0 || !epoch_jd || !t || !delta || !out)))
        return fail(BQP_E_ARG, "bad buffers");
    int rc = set_device(ctx);
    if (rc) return rc;
    if ((rc = frame_prepare_dev(ctx, n, epoch_jd, 0.0, t, t))) return rc;
    cudaError_t e = launch_rhs(ctx->d_tab, ctx->ncells, ctx->use_smem, force_params(ctx), n, equ, seg_t0,
                               epoch_jd, t, delta, ballistic, ctx->cfg.am_ratio, ctx->cfg.cd, out, ctx->stream);
    return e == cudaSuccess ? 0 : cuda_fail(e, "k_rhs launch");
}

int bqp_rhs_eval(bqp_ctx* ctx, int64_t n, const double* equ, const double* seg_t0, const double* epoch_jd,
                 const double* t, const double* delta, const double* ballistic, double* out) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    if (n < 0 || (n > 0 && (!equ || !seg_t0 || !epoch_jd || !t || !delta || !out)))
        return fail(BQP_E_ARG, "bad buffers");
    if (n == 0) return 0;
    int rc = set_device(ctx);
    if (rc) return rc;
    if ((rc = frame_prepare_host(ctx, n, epoch_jd, t, t))) return rc;
    const size_t b6 = (size_t)n * 6 * sizeof(double), b1 = (size_t)n * sizeof(double);
    double *de = nullptr, *dt0 = nullptr, *djd = nullptr, *dt = nullptr, *dd = nullptr, *db = nullptr,
           *dout = nullptr;
    for (int pass = 0; pass < 2; ++pass) {
        Carve cv{pass ? (char*)ctx->d_ws : nullptr};
        de = cv.take<double>((size_t)n * 6);
        dt0 = cv.take<double>((size_t)n);
        djd = cv.take<double>((size_t)n);
        dt = cv.take<double>((size_t)n);
        dd = cv.take<double>((size_t)n * 6);
        db = ballistic ? cv.take<double>((size_t)n * 2) : nullptr;
        dout = cv.take<double>((size_t)n * 6);
        if (!pass && (rc = ensure_ws(ctx, cv.off))) return rc;
    }
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(de, equ, b6, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt0, seg_t0, b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(djd, epoch_jd, b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dt, t, b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dd, delta, b6, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && db) e = cudaMemcpyAsync(db, ballistic, 2 * b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = launch_rhs(ctx->d_tab, ctx->ncells, ctx->use_smem, force_params(ctx), n, de, dt0, djd, dt, dd, db,
                       ctx->cfg.am_ratio, ctx->cfg.cd, dout, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, b6, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? 0 : cuda_fail(e, "bqp_rhs_eval");
}

int bqp_propagate_final_device(bqp_ctx* ctx, int64_t n, const double* in, int32_t input_equ,
                               const double* epoch_jd, double t0, const double* tf, const double* ballistic,
                               double* out, int32_t* status, int64_t* steps, int64_t* evals) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    int rc = check_prop_args(n, in, epoch_jd, t0, tf, out, status);
    if (rc) return rc;
    if (n == 0) return 0;
    if ((rc = set_device(ctx))) return rc;
    return launch_prop(ctx, n, in, input_equ, epoch_jd, t0, tf, ballistic, 0, nullptr, 0, out, status, steps,
                       evals);
}

int bqp_propagate_final(bqp_ctx* ctx, int64_t n, const double* in, int32_t input_equ, const double* epoch_jd,
                        double t0, const double* tf, const double* ballistic, double* out, int32_t* status,
                        int64_t* steps, int64_t* evals) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    int rc = check_prop_args(n, in, epoch_jd, t0, tf, out, status);
    if (rc) return rc;
    if (n == 0) return 0;
    if ((rc = set_device(ctx))) return rc;
    const size_t b6 = (size_t)n * 6 * sizeof(double), b1 = (size_t)n * sizeof(double);
    double *din = nullptr, *dep = nullptr, *dtf = nullptr, *db = nullptr, *dout = nullptr;
    int32_t* dst = nullptr;
    int64_t *dsteps = nullptr, *devals = nullptr;
    for (int pass = 0; pass < 2; ++pass) {
        Carve cv{pass ? (char*)ctx->d_ws : nullptr};
        din = cv.take<double>((size_t)n * 6);
        dep = cv.take<double>((size_t)n);
        dtf = cv.take<double>((size_t)n);
        db = ballistic ? cv.take<double>((size_t)n * 2) : nullptr;
        dout = cv.take<double>((size_t)n * 6);
        dst = cv.take<int32_t>((size_t)n);
        dsteps = cv.take<int64_t>((size_t)n);
        devals = cv.take<int64_t>((size_t)n);
        if (!pass && (rc = ensure_ws(ctx, cv.off))) return rc;
    }
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(din, in, b6, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dep, epoch_jd, b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dtf, tf, b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && db) e = cudaMemcpyAsync(db, ballistic, 2 * b1, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "bqp_propagate_final H2D");
    rc = launch_prop(ctx, n, din, input_equ, dep, t0, dtf, db, 0, nullptr, 0, dout, dst, dsteps, devals);
    if (rc) return rc;
    e = cudaMemcpyAsync(out, dout, b6, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(status, dst, (size_t)n * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && steps) e = cudaMemcpyAsync(steps, dsteps, b1, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && evals) e = cudaMemcpyAsync(evals, devals, b1, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? 0 : cuda_fail(e, "bqp_propagate_final");
}

int bqp_propagate_sampled_device(bqp_ctx* ctx, int64_t n, const double* in, int32_t input_equ,
                                 const double* epoch_jd, double t0, const double* tf, int32_t n_t,
                                 const double* t_eval, int32_t out_deltas, double* out, int32_t* status,
                                 int64_t* steps, int64_t* evals) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    int rc = check_prop_args(n, in, epoch_jd, t0, tf, out, status);
    if (rc) return rc;
    if (n_t <= 0 || !t_eval) return fail(BQP_E_ARG, "t_eval must be a non-empty array");
    if (n == 0) return 0;
    if ((rc = set_device(ctx))) return rc;
    return launch_prop(ctx, n, in, input_equ, epoch_jd, t0, tf, nullptr, n_t, t_eval,
                       out_deltas ? 2 : 1, out, status, steps, evals);
}

int bqp_propagate_sampled(bqp_ctx* ctx, int64_t n, const double* in, int32_t input_equ, const double* epoch_jd,
                          double t0, const double* tf, int32_t n_t, const double* t_eval, int32_t out_deltas,
                          double* out, int32_t* status, int64_t* steps, int64_t* evals) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    int rc = check_prop_args(n, in, epoch_jd, t0, tf, out, status);
    if (rc) return rc;
    if ((rc = check_grid(n_t, t_eval))) return rc;
    if (t_eval[0] < t0) return fail(BQP_E_ARG, "t_eval starts before t0");
    for (int64_t i = 0; i < n; ++i)
        if (!(tf[i] >= t_eval[n_t - 1])) return fail(BQP_E_ARG, "t_eval ends after tf[%lld]", (long long)i);
    if (n == 0) return 0;
    if ((rc = set_device(ctx))) return rc;
    const size_t b6 = (size_t)n * 6 * sizeof(double), b1 = (size_t)n * sizeof(double);
    const size_t bo = (size_t)n * n_t * 6 * sizeof(double);
    double *din = nullptr, *dep = nullptr, *dtf = nullptr, *dte = nullptr, *dout = nullptr;
    int32_t* dst = nullptr;
    int64_t *dsteps = nullptr, *devals = nullptr;
    for (int pass = 0; pass < 2; ++pass) {
        Carve cv{pass ? (char*)ctx->d_ws : nullptr};
        din = cv.take<double>((size_t)n * 6);
        dep = cv.take<double>((size_t)n);
        dtf = cv.take<double>((size_t)n);
        dte = cv.take<double>((size_t)n_t);
        dout = cv.take<double>((size_t)n * n_t * 6);
        dst = cv.take<int32_t>((size_t)n);
        dsteps = cv.take<int64_t>((size_t)n);
        devals = cv.take<int64_t>((size_t)n);
        if (!pass && (rc = ensure_ws(ctx, cv.off))) return rc;
    }
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(din, in, b6, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dep, epoch_jd, b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dtf, tf, b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dte, t_eval, (size_t)n_t * 8, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "bqp_propagate_sampled H2D");
    rc = launch_prop(ctx, n, din, input_equ, dep, t0, dtf, nullptr, n_t, dte, out_deltas ? 2 : 1, dout, dst,
                     dsteps, devals);
    if (rc) return rc;
    e = cudaMemcpyAsync(out, dout, bo, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(status, dst, (size_t)n * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && steps) e = cudaMemcpyAsync(steps, dsteps, b1, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && evals) e = cudaMemcpyAsync(evals, devals, b1, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? 0 : cuda_fail(e, "bqp_propagate_sampled");
}

int bqp_utc_jd(int64_t n, const double* jd0, const double* t, double* out) {
    if (n < 0 || (n > 0 && (!jd0 || !t || !out))) return fail(BQP_E_ARG, "bad buffers");
    for (int64_t i = 0; i < n; ++i) out[i] = utc_jd_at(jd0[i], t[i]);
    return 0;
}

int bqp_eci_to_equinoctial(int64_t n, const double* eci, double* equ, int32_t* ok) {
    if (n < 0 || (n > 0 && (!eci || !equ))) return fail(BQP_E_ARG, "bad buffers");
    for (int64_t i = 0; i < n; ++i) {
        bool good = eci_to_equinoctial(eci + 6 * i, equ + 6 * i);
        if (ok) ok[i] = good ? 1 : 0;
    }
    return 0;
}

int bqp_equinoctial_to_eci(int64_t n, const double* equ, const double* tof, double* eci) {
    if (n < 0 || (n > 0 && (!equ || !eci))) return fail(BQP_E_ARG, "bad buffers");
    for (int64_t i = 0; i < n; ++i) equinoctial_to_eci(equ + 6 * i, tof ? tof[i] : 0.0, eci + 6 * i);
    return 0;
}

int bqp_kep_to_eci(int64_t n, const double* kep, double* eci) {
    if (n < 0 || (n > 0 && (!kep || !eci))) return fail(BQP_E_ARG, "bad buffers");
    for (int64_t i = 0; i < n; ++i) kep2eci(kep + 6 * i, eci + 6 * i);
    return 0;
}

int bqp_eci_to_kep(int64_t n, const double* eci, double* kep) {
    if (n < 0 || (n > 0 && (!eci || !kep))) return fail(BQP_E_ARG, "bad buffers");
    for (int64_t i = 0; i < n; ++i) eci2kep(eci + 6 * i, kep + 6 * i);
    return 0;
}

}  // extern "C"

// ======================================================================
// Allocation-free final-state propagation (bqp_propagate_final_noalloc).
//
// For callers that cannot allocate device memory while they propagate: the
// staging buffers of the host-buffer call live in one fixed array compiled
// into the library instead of the context's growable workspace.  In host
// code `g_noalloc_scratch` is only the runtime's stand-in for that array; its
// device address comes from cudaGetSymbolAddress, looked up once per device
// with that device current, and only that address is handed to the kernel.
namespace {

constexpr size_t round256(size_t x) { return (x + 255) & ~(size_t)255; }

// Bytes one call carves for n rows, in carve order: work-queue counter;
// inputs (state, epoch, final time, ballistic pair); outputs (state, status,
// steps, evaluations).  Every array starts on a 256-byte boundary, as Carve
// places them.
constexpr size_t noalloc_bytes(size_t n) {
    return round256(sizeof(unsigned long long)) + round256(n * 6 * sizeof(double)) +
           2 * round256(n * sizeof(double)) + round256(n * 2 * sizeof(double)) +
           round256(n * 6 * sizeof(double)) + round256(n * sizeof(int32_t)) + 2 * round256(n * sizeof(int64_t));
}

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[noalloc_bytes(BQP_NOALLOC_MAX_TRAJ)];

namespace {

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;  // serialises the calls; guards g_noalloc_base
unsigned char* g_noalloc_base[kNoallocMaxDevices] = {};

// Device address of the scratch array on the current device (which the
// caller has made `device`), looked up on the first call on that device.
int noalloc_base(int device, unsigned char** out) {
    if (device < 0 || device >= kNoallocMaxDevices)
        return fail(BQP_E_ARG, "device %d is beyond the %d devices the no-allocation path supports", device,
                    kNoallocMaxDevices);
    if (!g_noalloc_base[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
        g_noalloc_base[device] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_base[device];
    return 0;
}

}  // namespace

extern "C" {

int bqp_propagate_final_noalloc(bqp_ctx* ctx, int64_t n, const double* in, int32_t input_equ,
                                const double* epoch_jd, double t0, const double* tf, const double* ballistic,
                                double* out, int32_t* status, int64_t* steps, int64_t* evals) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    // this path runs the persistent kernel on the FP64 field; a context set
    // up for a form only the stage-synchronous engine has is refused, not
    // run in plain FP64
    if (ctx->cfg.split_degree || ctx->cfg.surrogate || ctx->cfg.drag_fp32 || (ctx->cfg.force_flags & BQP_FORCE_SRP) ||
        ctx->frame)
        return fail(BQP_E_UNSUPPORTED,
                    "the no-allocation entry point runs plain FP64 without SRP in the GMST frame only; this context "
                    "is configured for %s",
                    ctx->cfg.surrogate ? "the learned surrogate"
                    : ctx->cfg.split_degree ? "split precision"
                    : ctx->cfg.drag_fp32 ? "the FP32 density"
                    : ctx->frame ? "the IAU 2006/2000A frame (segments built per call)"
                                 : "binary-eclipse SRP");
    int rc = check_prop_args(n, in, epoch_jd, t0, tf, out, status);
    if (rc) return rc;
    if (n > BQP_NOALLOC_MAX_TRAJ)
        return fail(BQP_E_ARG, "n = %lld rows exceeds the no-allocation limit of %d rows", (long long)n,
                    BQP_NOALLOC_MAX_TRAJ);
    if (n == 0) return 0;
    if ((rc = set_device(ctx))) return rc;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    unsigned char* base = nullptr;
    if ((rc = noalloc_base(ctx->device, &base))) return rc;

    Carve cv{reinterpret_cast<char*>(base)};
    unsigned long long* queue = cv.take<unsigned long long>(1);
    double* din = cv.take<double>((size_t)n * 6);
    double* dep = cv.take<double>((size_t)n);
    double* dtf = cv.take<double>((size_t)n);
    double* db = cv.take<double>((size_t)n * 2);
    double* dout = cv.take<double>((size_t)n * 6);
    int32_t* dst = cv.take<int32_t>((size_t)n);
    int64_t* dsteps = cv.take<int64_t>((size_t)n);
    int64_t* devals = cv.take<int64_t>((size_t)n);
    if (cv.off > sizeof(g_noalloc_scratch))
        return fail(BQP_E_ARG, "no-allocation staging of %zu bytes exceeds the %zu-byte array", cv.off,
                    sizeof(g_noalloc_scratch));

    const size_t b6 = (size_t)n * 6 * sizeof(double), b1 = (size_t)n * sizeof(double);
    cudaStream_t s = ctx->stream;
    // the work-queue counter is the one thing that must start at zero; every
    // output row is written by the kernel (finished, failed or drained)
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(din, in, b6, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dep, epoch_jd, b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dtf, tf, b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && ballistic) e = cudaMemcpyAsync(db, ballistic, 2 * b1, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "bqp_propagate_final_noalloc H2D");

    PropArgs A{};
    A.n = n;
    A.in = din;
    A.input_equinoctial = input_equ;
    A.epoch = dep;
    A.t0 = t0;
    A.tf = dtf;
    A.ballistic = ballistic ? db : nullptr;
    A.am0 = ctx->cfg.am_ratio;
    A.cd0 = ctx->cfg.cd;
    A.t_eval = nullptr;
    A.n_t = 0;
    A.out_mode = 0;
    A.out = dout;
    A.status = dst;
    A.steps = dsteps;
    A.evals = devals;
    A.queue = queue;
    A.gtab = ctx->d_tab;
    A.ncells = ctx->ncells;
    A.use_smem = ctx->use_smem;
    A.force = force_params(ctx);
    // the sweep fits are built with the context and rebuilt by the calls that
    // change them; if they are not current the quadrature runs instead (the
    // same densities within the fits' 1e-13), never stale fits
    if (!ctx->fit2_built) A.force.fit2 = nullptr;
    A.ctrl = ctrl_params(ctx);
    // event create/record allocate no device memory
    cudaEvent_t ev[2] = {nullptr, nullptr};
    if (ctx->profile) {
        cudaEventCreate(&ev[0]);
        cudaEventCreate(&ev[1]);
        cudaEventRecord(ev[0], s);
    }
    e = launch_propagate(A, ctx->cfg.method, 256, 0, s);
    if (ctx->profile) {
        cudaEventRecord(ev[1], s);
        float ms = 0.0f;
        if (e == cudaSuccess && cudaEventSynchronize(ev[1]) == cudaSuccess &&
            cudaEventElapsedTime(&ms, ev[0], ev[1]) == cudaSuccess) {
            ctx->times.ms[kKcPersistent] += ms;
            ctx->times.launches[kKcPersistent] += 1;
        }
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
    }
    if (e != cudaSuccess) return cuda_fail(e, "k_propagate launch (no-allocation path)");

    e = cudaMemcpyAsync(out, dout, b6, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(status, dst, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && steps) e = cudaMemcpyAsync(steps, dsteps, b1, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && evals) e = cudaMemcpyAsync(evals, devals, b1, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? 0 : cuda_fail(e, "bqp_propagate_final_noalloc");
}

}  // extern "C"

// ======================================================================
// Sigma-point covariance propagation (sigma.cu).
namespace {

struct SigmaBufs {
    double *rows, *row_epoch, *row_tf, *row_bal, *out_rows, *offsets, *wm, *wc;
    int32_t* row_status;
    int64_t* row_evals;
};

void carve_sigma(Carve& cv, int64_t n, int S, bool bal, SigmaBufs& B) {
    const size_t m = (size_t)n * S;
    B.rows = cv.take<double>(m * 6);
    B.row_epoch = cv.take<double>(m);
    B.row_tf = cv.take<double>(m);
    B.row_bal = bal ? cv.take<double>(m * 2) : nullptr;
    B.out_rows = cv.take<double>(m * 6);
    B.row_status = cv.take<int32_t>(m);
    B.row_evals = cv.take<int64_t>(m);
    B.offsets = cv.take<double>(7 * 6);
    B.wm = cv.take<double>(13);
    B.wc = cv.take<double>(13);
}

// Generation -> propagation of n * S rows -> recombination, all on ctx's
// stream; inputs and outputs are device pointers, B in the workspace.
int sigma_run(bqp_ctx* ctx, int64_t n, const SigmaSet& SS, int32_t set, const SigmaBufs& B, const double* mean,
              const double* cov, const double* epoch, double t0, const double* tf, const double* bal,
              double* mean_out, double* cov_out, int32_t* status, int64_t* evals) {
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(B.offsets, SS.offsets, sizeof SS.offsets, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(B.wm, SS.wm, sizeof SS.wm, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(B.wc, SS.wc, sizeof SS.wc, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = launch_sigma_gen(n, set == BQP_SIGMA_JULIER7 ? 0 : 1, SS.scale, B.offsets, mean, cov, epoch, tf, bal,
                             B.rows, B.row_epoch, B.row_tf, bal ? B.row_bal : nullptr, status, s);
    if (e != cudaSuccess) return cuda_fail(e, "sigma-point generation");
    int rc = launch_prop(ctx, n * SS.points, B.rows, 0, B.row_epoch, t0, B.row_tf, bal ? B.row_bal : nullptr, 0,
                         nullptr, 0, B.out_rows, B.row_status, nullptr, B.row_evals);
    if (rc) return rc;
    e = launch_sigma_recombine(n, SS.points, B.wm, B.wc, B.out_rows, B.row_status, B.row_evals, mean_out, cov_out,
                               status, evals, s);
    return e == cudaSuccess ? 0 : cuda_fail(e, "sigma-point recombination");
}

int check_sigma_args(const bqp_ctx* ctx, int64_t n, const double* mean, const double* cov, const double* epoch,
                     double t0, const double* tf, const double* mean_out, const double* cov_out,
                     const int32_t* status) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    if (n < 0) return fail(BQP_E_ARG, "n must be >= 0");
    if (n > 0 && (!mean || !cov || !epoch || !tf || !mean_out || !cov_out || !status))
        return fail(BQP_E_ARG, "null buffer");
    if (!std::isfinite(t0)) return fail(BQP_E_ARG, "t0 must be finite");
    return 0;
}

}  // namespace

extern "C" {

int bqp_sigma_weights(int32_t set, double alpha, double beta, double kappa, int32_t* points, double* wm,
                      double* wc, double* offsets) {
    SigmaSet SS;
    int rc = sigma_set(set, alpha, beta, kappa, SS);
    if (rc) return rc;
    if (points) *points = SS.points;
    for (int p = 0; p < SS.points; ++p) {
        if (wm) wm[p] = SS.wm[p];
        if (wc) wc[p] = SS.wc[p];
    }
    if (offsets)
        for (int k = 0; k < 42; ++k) offsets[k] = SS.offsets[k];
    return 0;
}

int bqp_sigma_propagate_device(bqp_ctx* ctx, int64_t n, const double* mean, const double* cov, int32_t set,
                               double alpha, double beta, double kappa, const double* epoch_jd, double t0,
                               const double* tf, const double* ballistic, double* mean_out, double* cov_out,
                               int32_t* status, int64_t* evals) {
    int rc = check_sigma_args(ctx, n, mean, cov, epoch_jd, t0, tf, mean_out, cov_out, status);
    if (rc) return rc;
    SigmaSet SS;
    if ((rc = sigma_set(set, alpha, beta, kappa, SS))) return rc;
    if (n == 0) return 0;
    if ((rc = set_device(ctx))) return rc;
    SigmaBufs B{};
    for (int pass = 0; pass < 2; ++pass) {
        Carve cv{pass ? (char*)ctx->d_ws : nullptr};
        carve_sigma(cv, n, SS.points, ballistic != nullptr, B);
        if (!pass && (rc = ensure_ws(ctx, cv.off))) return rc;
    }
    return sigma_run(ctx, n, SS, set, B, mean, cov, epoch_jd, t0, tf, ballistic, mean_out, cov_out, status,
                     evals);
}

int bqp_sigma_propagate(bqp_ctx* ctx, int64_t n, const double* mean, const double* cov, int32_t set,
                        double alpha, double beta, double kappa, const double* epoch_jd, double t0,
                        const double* tf, const double* ballistic, double* mean_out, double* cov_out,
                        int32_t* status, int64_t* evals) {
    int rc = check_sigma_args(ctx, n, mean, cov, epoch_jd, t0, tf, mean_out, cov_out, status);
    if (rc) return rc;
    SigmaSet SS;
    if ((rc = sigma_set(set, alpha, beta, kappa, SS))) return rc;
    if (n == 0) return 0;
    if ((rc = set_device(ctx))) return rc;
    SigmaBufs B{};
    double *dm = nullptr, *dc = nullptr, *dep = nullptr, *dtf = nullptr, *db = nullptr, *dmo = nullptr,
           *dco = nullptr;
    int32_t* dst = nullptr;
    int64_t* dev = nullptr;
    const size_t b1 = (size_t)n * sizeof(double);
    for (int pass = 0; pass < 2; ++pass) {
        Carve cv{pass ? (char*)ctx->d_ws : nullptr};
        carve_sigma(cv, n, SS.points, ballistic != nullptr, B);
        dm = cv.take<double>((size_t)n * 6);
        dc = cv.take<double>((size_t)n * 36);
        dep = cv.take<double>((size_t)n);
        dtf = cv.take<double>((size_t)n);
        db = ballistic ? cv.take<double>((size_t)n * 2) : nullptr;
        dmo = cv.take<double>((size_t)n * 6);
        dco = cv.take<double>((size_t)n * 36);
        dst = cv.take<int32_t>((size_t)n);
        dev = cv.take<int64_t>((size_t)n);
        if (!pass && (rc = ensure_ws(ctx, cv.off))) return rc;
    }
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(dm, mean, 6 * b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dc, cov, 36 * b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dep, epoch_jd, b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dtf, tf, b1, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && db) e = cudaMemcpyAsync(db, ballistic, 2 * b1, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "bqp_sigma_propagate H2D");
    rc = sigma_run(ctx, n, SS, set, B, dm, dc, dep, t0, dtf, db, dmo, dco, dst, dev);
    if (rc) return rc;
    e = cudaMemcpyAsync(mean_out, dmo, 6 * b1, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(cov_out, dco, 36 * b1, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(status, dst, (size_t)n * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && evals) e = cudaMemcpyAsync(evals, dev, b1, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? 0 : cuda_fail(e, "bqp_sigma_propagate");
}

}  // extern "C"

// ======================================================================
// Tensor-core GEMM of the gravity surrogate, exported for its tests.
extern "C" int bqp_gemm_bf16_device(int64_t m, int64_t n, int64_t k, const void* a, const void* b, float* c,
                                    void* stream) {
    if (m < 0 || n < 0 || k < 0 || (m && n && k && (!a || !b || !c))) return fail(BQP_E_ARG, "bad GEMM arguments");
    if (m % 128 || n % 256 || k % 64)
        return fail(BQP_E_ARG, "GEMM shape %lld x %lld x %lld: M must be a multiple of 128, N of 256, K of 64",
                    (long long)m, (long long)n, (long long)k);
    int* derr = nullptr;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMallocAsync(&derr, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(derr, 0, sizeof(int), s);
    if (e == cudaSuccess) e = launch_gemm_bf16(m, n, k, a, b, c, derr, s);
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (derr) cudaFreeAsync(derr, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "bqp_gemm_bf16");
    if (herr) return fail(BQP_E_CUDA, "tensor-core GEMM: an mbarrier wait timed out");
    return 0;
}

// ======================================================================
// Learned gravity surrogate (surrogate.cu).
namespace {

GravTable plain_table(const bqp_ctx* ctx) {
    GravTable T{};
    T.tab = ctx->d_tab;
    T.order = ctx->cfg.order;
    T.ls = 0;
    T.bytes = (uint32_t)ctx->tab_bytes;
    T.in_smem = T.bytes <= kSmemLimit ? 1 : 0;
    return T;
}

int ensure_low_table(bqp_ctx* ctx) {
    if (ctx->d_tab_low) return 0;
    if (ctx->parsed_order < BQP_SURROGATE_DEGREE)
        return fail(BQP_E_ARG, "the surrogate needs a field of degree > %d", BQP_SURROGATE_DEGREE);
    std::vector<double> tab = build_gravity_table(ctx->coeffs, BQP_SURROGATE_DEGREE);
    ctx->low_bytes = (uint32_t)(tab.size() * sizeof(double));
    cudaError_t e = cudaMalloc(&ctx->d_tab_low, ctx->low_bytes);
    if (e == cudaSuccess) e = cudaMemcpy(ctx->d_tab_low, tab.data(), ctx->low_bytes, cudaMemcpyHostToDevice);
    return e == cudaSuccess ? 0 : cuda_fail(e, "surrogate low-degree table");
}

GravTable low_table(const bqp_ctx* ctx) {
    GravTable T{};
    T.tab = ctx->d_tab_low;
    T.order = BQP_SURROGATE_DEGREE;
    T.ls = 0;
    T.bytes = ctx->low_bytes;
    T.in_smem = 1;
    return T;
}

int surrogate_ready(bqp_ctx* ctx, bool need_trained);

// The propagation's view of the trained surrogate (pipeline gravity stage).
int surrogate_stage_args(bqp_ctx* ctx, SurrogateRef& S) {
    int rc = surrogate_ready(ctx, true);
    if (rc) return rc;
    if (ctx->cfg.order <= BQP_SURROGATE_DEGREE)
        return fail(BQP_E_ARG, "the surrogate replaces degrees above %d; the order is %d", BQP_SURROGATE_DEGREE,
                    ctx->cfg.order);
    Model& M = *ctx->sur;
    S.P = M.P;
    S.Wtile = M.Wtile;
    S.R = M.scale.R;
    S.r_mid = M.scale.r_mid;
    S.r_half = M.scale.r_half;
    S.sigma = M.sigma;
    S.err = M.derr;
    S.low = low_table(ctx);
    S.full = grav_table(ctx);
    S.check = ctx->cfg.surrogate_check;
    return 0;
}

int surrogate_ready(bqp_ctx* ctx, bool need_trained) {
    if (!ctx) return fail(BQP_E_ARG, "null ctx");
    int rc = set_device(ctx);
    if (rc) return rc;
    if ((rc = ensure_low_table(ctx))) return rc;
    if (!ctx->sur) ctx->sur = new Model();
    if (need_trained && !ctx->sur->trained) return fail(BQP_E_ARG, "the surrogate has not been trained or loaded");
    return 0;
}

}  // namespace

extern "C" {

int bqp_surrogate_infer_device(bqp_ctx* ctx, int64_t n, const double* pos_km, double* acc, int32_t add_low);

int bqp_surrogate_train(bqp_ctx* ctx, int64_t samples, int32_t epochs, int32_t batch, double lr, uint64_t seed,
                        double* loss_per_epoch) {
    int rc = surrogate_ready(ctx, false);
    if (rc) return rc;
    if (ctx->cfg.order <= BQP_SURROGATE_DEGREE)
        return fail(BQP_E_ARG, "the surrogate learns degrees above %d; the context's order is %d", BQP_SURROGATE_DEGREE,
                    ctx->cfg.order);
    if (samples < 1024 || epochs < 1 || batch < 128 || batch % 128 || batch > 65536 || !(lr > 0.0))
        return fail(BQP_E_ARG, "samples >= 1024, epochs >= 1, batch a multiple of 128 up to 65536, lr > 0");
    const GravTable full = plain_table(ctx), low = low_table(ctx);
    cudaStream_t s = ctx->stream;
    FieldFn ffull = [&](int64_t n, const double* pos, double* acc) {
        return launch_gravity(full, n, pos, acc, nullptr, s, 256, 4);
    };
    FieldFn flow = [&](int64_t n, const double* pos, double* acc) {
        return launch_gravity(low, n, pos, acc, nullptr, s, 256, 4);
    };
    TrainArgs a{samples, epochs, batch, lr, seed};
    cudaError_t e = train(*ctx->sur, a, ffull, flow, s, loss_per_epoch);
    if (e == cudaErrorLaunchTimeout) return fail(BQP_E_CUDA, "surrogate training: a tensor-core wait timed out");
    return e == cudaSuccess ? 0 : cuda_fail(e, "surrogate training");
}

int bqp_surrogate_infer(bqp_ctx* ctx, int64_t n, const double* pos_km, double* acc, int32_t add_low) {
    int rc = surrogate_ready(ctx, true);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!pos_km || !acc))) return fail(BQP_E_ARG, "bad buffers");
    if (n == 0) return 0;
    double *dp = nullptr, *da = nullptr;
    for (int pass = 0; pass < 2; ++pass) {
        Carve cv{pass ? (char*)ctx->d_ws : nullptr};
        dp = cv.take<double>((size_t)n * 3);
        da = cv.take<double>((size_t)n * 3);
        if (!pass && (rc = ensure_ws(ctx, cv.off))) return rc;
    }
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(dp, pos_km, (size_t)n * 24, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "bqp_surrogate_infer H2D");
    if ((rc = bqp_surrogate_infer_device(ctx, n, dp, da, add_low))) return rc;
    e = cudaMemcpyAsync(acc, da, (size_t)n * 24, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? 0 : cuda_fail(e, "bqp_surrogate_infer");
}

int bqp_surrogate_infer_device(bqp_ctx* ctx, int64_t n, const double* pos_km, double* acc, int32_t add_low) {
    int rc = surrogate_ready(ctx, true);
    if (rc) return rc;
    if (n < 0 || (n > 0 && (!pos_km || !acc))) return fail(BQP_E_ARG, "bad buffers");
    if (n == 0) return 0;
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaSuccess;
    const bool low = (add_low & 1) != 0, unfused = (add_low & 2) != 0;
    if (low) e = launch_gravity(low_table(ctx), n, pos_km, acc, nullptr, s, 256, 4);
    else e = cudaMemsetAsync(acc, 0, (size_t)n * 24, s);
    if (e == cudaSuccess) {
        if (unfused) {
            e = infer(*ctx->sur, n, pos_km, acc, 1, s);
        } else {
            Model& M = *ctx->sur;
            e = cudaMemsetAsync(M.derr, 0, sizeof(int), s);
            if (e == cudaSuccess) e = infer_fused(M, n, pos_km, acc, M.derr, s);
        }
    }
    return e == cudaSuccess ? 0 : cuda_fail(e, "bqp_surrogate_infer_device");
}

int bqp_surrogate_params(bqp_ctx* ctx, float* params, double* sigma) {
    int rc = surrogate_ready(ctx, true);
    if (rc) return rc;
    if (!params || !sigma) return fail(BQP_E_ARG, "null argument");
    cudaError_t e = cudaMemcpy(params, ctx->sur->P, sg::kParams * 4, cudaMemcpyDeviceToHost);
    *sigma = ctx->sur->sigma;
    return e == cudaSuccess ? 0 : cuda_fail(e, "bqp_surrogate_params");
}

int bqp_surrogate_set_params(bqp_ctx* ctx, const float* params, double sigma) {
    int rc = surrogate_ready(ctx, false);
    if (rc) return rc;
    if (!params || !(sigma > 0.0)) return fail(BQP_E_ARG, "null parameters or sigma <= 0");
    cudaError_t e = upload_params(*ctx->sur, params, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    ctx->sur->sigma = sigma;
    return e == cudaSuccess ? 0 : cuda_fail(e, "bqp_surrogate_set_params");
}

int bqp_surrogate_grad(bqp_ctx* ctx, int32_t batch, const float* params, const float* x, const float* t,
                       float* grad, double* loss, float* y) {
    int rc = surrogate_ready(ctx, false);
    if (rc) return rc;
    if (batch < 128 || batch % 128 || batch > 65536 || !params || !x || !t || !grad || !loss)
        return fail(BQP_E_ARG, "batch a multiple of 128 up to 65536 and non-null buffers");
    Model& M = *ctx->sur;
    cudaStream_t s = ctx->stream;
    cudaError_t e = upload_params(M, params, s);
    if (e == cudaSuccess) e = M.alloc_batch(batch);
    if (e == cudaSuccess && !M.G) e = cudaMalloc(&M.G, sg::kParams * 4);
    M.dsum = reinterpret_cast<double*>(reinterpret_cast<char*>(M.derr) + 16);
    if (e == cudaSuccess) e = cudaMemcpyAsync(M.xb, x, (size_t)batch * 16, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(M.tb, t, (size_t)batch * 12, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(M.derr, 0, 32, s);
    if (e == cudaSuccess) e = forward_backward(M, batch, true, s);
    double lsum = 0.0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(grad, M.G, sg::kParams * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&lsum, M.dsum, 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && y) e = cudaMemcpyAsync(y, M.y, (size_t)batch * 12, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    *loss = lsum / (3.0 * batch);
    return e == cudaSuccess ? 0 : cuda_fail(e, "bqp_surrogate_grad");
}

}  // extern "C"
