// SOLFSMY / DTCFILE parsing and the exospheric-temperature bounds of a span
// of days (host code).  The checks follow jb_rs/src/drivers.rs: release
// header, 12 fields per SOLFSMY row with finite values and an integer Julian
// day equal to the row's Gregorian date, "DTC year doy" plus 24 integer
// hourly values per DTCFILE row, both files consecutive days without gaps or
// repeats (1025-1240), and the DTC coverage inside the SOLFSMY coverage
// (392-410).
#include "space_weather.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace bqp {

namespace {

constexpr int64_t kJdnOfOrdinalZero = 1721426;  // Julian day number of 0001-01-01 (proleptic Gregorian)

// Splits a (pointer, length) buffer into lines.
class LineReader {
   public:
    LineReader(const char* p, int64_t n) : p_(p), end_(p + (n > 0 ? n : 0)) {}
    bool next(std::string* line) {
        if (p_ >= end_) return false;
        const char* q = static_cast<const char*>(std::memchr(p_, '\n', (size_t)(end_ - p_)));
        if (!q) q = end_;
        line->assign(p_, q);
        p_ = q < end_ ? q + 1 : end_;
        return true;
    }

   private:
    const char* p_;
    const char* end_;
};

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\f' || c == '\v'; }

std::vector<std::string> tokens(const std::string& s) {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < s.size()) {
        while (i < s.size() && is_space(s[i])) ++i;
        size_t j = i;
        while (j < s.size() && !is_space(s[j])) ++j;
        if (j > i) out.emplace_back(s, i, j - i);
        i = j;
    }
    return out;
}

bool blank(const std::string& s) {
    return std::all_of(s.begin(), s.end(), [](char c) { return is_space(c); });
}

char first_char(const std::string& s) {
    for (char c : s)
        if (!is_space(c)) return c;
    return 0;
}

bool to_int(const std::string& t, int64_t lo, int64_t hi, int64_t* v) {
    if (t.empty()) return false;
    char* e = nullptr;
    errno = 0;
    const long long x = std::strtoll(t.c_str(), &e, 10);
    if (*e != 0 || errno != 0 || x < lo || x > hi) return false;
    *v = x;
    return true;
}

bool to_finite(const std::string& t, double* v) {
    if (t.empty() || t.find_first_of("xX") != std::string::npos) return false;  // decimal forms only
    char* e = nullptr;
    *v = std::strtod(t.c_str(), &e);
    return *e == 0 && std::isfinite(*v);
}

// Days since 0001-01-01 of (year, day of year); -1 for an invalid date.
int64_t day_ordinal(const std::string& ys, const std::string& ds) {
    int64_t y, d;
    if (!to_int(ys, 1, 2147483647, &y) || !to_int(ds, 1, 366, &d)) return -1;
    const bool leap = y % 4 == 0 && (y % 100 != 0 || y % 400 == 0);
    if (d > (leap ? 366 : 365)) return -1;
    const int64_t c = y - 1;
    return 365 * c + c / 4 - c / 100 + c / 400 + d - 1;
}

}  // namespace

std::string parse_space_weather(const char* solfsmy, int64_t solfsmy_len, const char* dtcfile, int64_t dtcfile_len,
                                SpaceWeather* out) {
    if (!solfsmy || !dtcfile || solfsmy_len < 0 || dtcfile_len < 0) return "missing file text";
    SpaceWeather sw;
    std::vector<int64_t> solar_ord, dtc_ord;
    std::string line;
    bool header = false;
    LineReader sol(solfsmy, solfsmy_len);
    for (int64_t ln = 1; sol.next(&line); ++ln) {
        if (blank(line)) continue;
        if (first_char(line) == '#') {
            if (!header) {
                header = true;
                const size_t at = line.find('#');
                if (line.compare(at, 33, "# F10, S10, M10, Y10 data release") != 0)
                    return "SOLFSMY release header is unrecognized";
            }
            continue;
        }
        const auto f = tokens(line);
        const std::string where = " (SOLFSMY line " + std::to_string(ln) + ")";
        if (f.size() != 12) return "expected 12 fields" + where;
        const int64_t ord = day_ordinal(f[0], f[1]);
        if (ord < 0) return "invalid calendar date" + where;
        double jd, v[8];
        if (!to_finite(f[2], &jd) || jd != std::floor(jd)) return "Julian day is not an integer noon key" + where;
        for (int k = 0; k < 8; ++k)
            if (!to_finite(f[3 + k], &v[k])) return "non-finite or non-numeric index" + where;
        if (jd != (double)(ord + kJdnOfOrdinalZero)) return "date and Julian day disagree" + where;
        if (!solar_ord.empty() && ord != solar_ord.back() + 1) return "rows missing, repeated or out of order" + where;
        if (sw.n_solar == 0) sw.first_jd = jd;
        sw.solar.insert(sw.solar.end(), v, v + 8);
        solar_ord.push_back(ord);
        ++sw.n_solar;
    }
    if (!header) return "SOLFSMY release header missing";
    if (sw.n_solar == 0) return "SOLFSMY has no data rows";

    LineReader dtc(dtcfile, dtcfile_len);
    for (int64_t ln = 1; dtc.next(&line); ++ln) {
        if (blank(line) || first_char(line) == '#') continue;
        const auto f = tokens(line);
        const std::string where = " (DTCFILE line " + std::to_string(ln) + ")";
        if (f.size() != 27 || f[0] != "DTC") return "expected DTC plus 26 fields" + where;
        const int64_t ord = day_ordinal(f[1], f[2]);
        if (ord < 0) return "invalid calendar date" + where;
        for (int h = 0; h < 24; ++h) {
            int64_t x;
            if (!to_int(f[3 + h], -2147483648LL, 2147483647LL, &x)) return "dTc is not a 32-bit integer" + where;
            sw.dtc.push_back((int32_t)x);
        }
        if (!dtc_ord.empty() && ord != dtc_ord.back() + 1) return "rows missing, repeated or out of order" + where;
        dtc_ord.push_back(ord);
        ++sw.n_dtc;
    }
    if (sw.n_dtc == 0) return "DTCFILE has no data rows";
    if (dtc_ord.front() < solar_ord.front() || dtc_ord.back() > solar_ord.back())
        return "DTCFILE coverage has no matching SOLFSMY calendar date";
    sw.dtc_first = (int32_t)(dtc_ord.front() - solar_ord.front());
    *out = std::move(sw);
    return "";
}

bool space_weather_tinf_range(const SpaceWeather& sw, double jd_lo, double jd_hi, double* tlo, double* thi) {
    // solar rows whose day a lookup in the span can land on
    int i0 = 5, i1 = sw.n_solar - 1;
    if (jd_lo != 0.0 || jd_hi != 0.0) {
        i0 = std::max(i0, (int)std::floor(std::floor(jd_lo + 0.5) - sw.first_jd));
        i1 = std::min(i1, (int)std::floor(std::floor(jd_hi + 0.5) - sw.first_jd));
    }
    double lo = 1e300, hi = -1e300, f10_lo = 1e300, f10_hi = -1e300;
    for (int i = i0; i <= i1; ++i) {
        const int r = i - sw.dtc_first;
        if (r < 0 || r >= sw.n_dtc) continue;
        const double* a = &sw.solar[(size_t)(i - 1) * 8];
        const double* m = &sw.solar[(size_t)(i - 2) * 8];
        const double* y = &sw.solar[(size_t)(i - 5) * 8];
        // interpolated dTc stays between the day's hourly values and the next day's first
        int32_t dmin = sw.dtc[(size_t)r * 24], dmax = dmin;
        for (int h = 0; h < 24 + (r + 1 < sw.n_dtc ? 1 : 0); ++h) {
            const int32_t v = sw.dtc[(size_t)r * 24 + h];
            dmin = std::min(dmin, v);
            dmax = std::max(dmax, v);
        }
        // the exospheric temperature before the diurnal factor and dTc (jb2008.rs)
        const double fn = std::fmin(std::pow(a[1] / 240.0, 0.25), 1.0);
        const double fsb = a[1] * fn + a[3] * (1.0 - fn);
        const double tsubc = 392.4 + 3.227 * fsb + 0.298 * (a[0] - a[1]) + 2.259 * (a[2] - a[3]) +
                             0.312 * (m[4] - m[5]) + 0.178 * (y[6] - y[7]);
        lo = std::fmin(lo, std::fmin(tsubc, tsubc * 1.31) + dmin);
        hi = std::fmax(hi, std::fmax(tsubc, tsubc * 1.31) + dmax);
        f10_lo = std::fmin(f10_lo, a[0]);
        f10_hi = std::fmax(f10_hi, a[0]);
    }
    if (!(hi >= lo)) return false;
    // the local-time / latitude / altitude correction is affine in F10 at each
    // point, so its extremes over the span sit at the span's extreme F10
    double cmin = 1e300, cmax = -1e300;
    for (double f10 : {f10_lo, f10_hi})
        for (int ih = 0; ih <= 480; ++ih)
            for (int ic = 0; ic <= 50; ++ic)
                for (int ia = 0; ia <= 60; ++ia) {
                    const double v = jb::dtc_correction(f10, ih * 0.05, ic * 0.02, 90.0 + ia * 50.0);
                    cmin = std::fmin(cmin, v);
                    cmax = std::fmax(cmax, v);
                }
    *tlo = lo + cmin - 10.0;
    *thi = hi + cmax + 10.0;
    return true;
}

}  // namespace bqp
