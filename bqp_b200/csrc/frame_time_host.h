// Host API of the IAU 2006/2000A frame chain and segment builder
// (frame_time.cpp).  Matrices are row-major double[9].
#pragma once
#include <cstdint>
#include <map>
#include <mutex>
#include <vector>

#include "frame_time.h"

namespace bqp {
namespace ft {

typedef double Mat3[9];

// ERFA-restated primitives (dates are two-part TT or UT1 Julian days).
void nut00a(double d1, double d2, double* dpsi, double* deps);
void nut06a(double d1, double d2, double* dpsi, double* deps);
double obl06(double d1, double d2);
void pfw06(double d1, double d2, double* gamb, double* phib, double* psib, double* epsa);
void pnm06a(double d1, double d2, Mat3 r);
double s06(double d1, double d2, double x, double y);
void xys06a(double d1, double d2, double* x, double* y, double* s);
void c2ixys(double x, double y, double s, Mat3 r);
double sp00(double d1, double d2);
void pom00(double xp, double yp, double sp, Mat3 r);
double era(double u1, double u2);
int utc_calendar_to_jd(int iy, int im, int id, int ihr, int imn, double sec, double* d1, double* d2);

// Earth-orientation records: per UTC day from `first_mjd`, five values each
// (x_p arcsec, y_p arcsec, UT1-UTC s, dX mas, dY mas) -- the layout of the
// reference's sealed eop_table.bin.  Empty: every value zero ("zero EOP").
struct Eop {
    int32_t first_mjd = 0;
    std::vector<double> rec;
    int32_t count() const { return (int32_t)(rec.size() / 5); }
    // false when the day is outside a non-empty table
    bool at(int32_t mjd, double out[5]) const;
};

// GCRS->ITRS at a UTC calendar instant plus `offset` seconds of TAI, by the
// fixture chain of chain.rs:140-297 (policy 0 zero EOP at the anchor, 1 the
// four-node Lagrange of `eop`).  r: R rounded to binary64; r_dd (optional):
// the pair's hi and lo parts, [2][9].  Returns 0, or < 0 on a bad instant or
// a missing EOP record.
int frame_matrix(int iy, int im, int id, int ihr, int imn, double sec, int policy, double offset,
                 const Eop& eop, Mat3 r, double* r_dd);
// R, Rdot, Rddot from the centred five-point stencil of step h
// (chain.rs:299-360), each rounded to binary64.
int frame_derivatives(int iy, int im, int id, int ihr, int imn, double sec, int policy, double h,
                      const Eop& eop, Mat3 r, Mat3 rdot, Mat3 rddot);

// A GCRS position, velocity and acceleration in ITRS through that stencil's
// R, Rdot, Rddot, summed in pairs (chain.rs transform_state).
int frame_transform_state(int iy, int im, int id, int ihr, int imn, double sec, int policy, double h,
                          const Eop& eop, const double* r, const double* v, const double* a, double* ro,
                          double* vo, double* ao);

// The segment authority over one EOP table (authority.rs:355-650).
class Authority {
public:
    explicit Authority(const Eop& eop);
    const FrameIntervals& intervals() const { return ivl_; }
    // Continuous TAI seconds of a UTC Julian day (one part); false outside.
    static bool tai_of_utc_jd(double jd, double* tai) { return tai_seconds_from_utc_jd(jd, tai); }
    // Build segment (j, k); false when its EOP nodes are missing.
    bool build(int32_t j, int64_t k, FrameSeg* out) const;
    // Segment holding `tai`, built once and kept; false outside the span.
    bool segment(double tai, int64_t* key, FrameSeg* out);
    // Every key whose segment holds an instant of [lo, hi], in order.
    void keys_between(double lo, double hi, std::vector<std::pair<int32_t, int64_t>>* out) const;
    // Build (and keep) the segments of `keys`, in parallel; returns the
    // subset that built, sorted, with their segments.
    void ensure(const std::vector<std::pair<int32_t, int64_t>>& keys, std::vector<int64_t>* built_keys,
                std::vector<FrameSeg>* built);

private:
    Eop eop_;
    FrameIntervals ivl_;
    std::mutex mu_;
    std::map<int64_t, FrameSeg> cache_;
    std::map<int64_t, bool> failed_;
};

}  // namespace ft
}  // namespace bqp
