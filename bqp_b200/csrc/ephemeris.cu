// "DUST" catalogue parsing (host code).  Layout: 48-byte little-endian header
// (4-byte magic "DUST", u32 version 1, u64 sample count, f64 first JD, f64
// last JD, f64 step in days, u8 body id, u8 epoch-scale tag 0-4, u8
// epoch-representation tag 0-2, five zero bytes), then samples x 3 f64.  The
// last JD must equal first + (samples - 1) x step as the producer rounds it,
// and every position must be finite.
#include "ephemeris.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace bqp {

namespace {

template <class T>
T read_le(const uint8_t* p) {
    T v;
    std::memcpy(&v, p, sizeof v);  // x86-64 and aarch64 hosts are little-endian
    return v;
}

}  // namespace

std::string parse_ephemeris(const uint8_t* b, int64_t len, int body, Ephemeris* out) {
    constexpr int64_t kHeader = 48;
    if (!b || len < kHeader) return "shorter than the 48-byte header";
    if (std::memcmp(b, "DUST", 4) != 0) return "magic is not DUST";
    if (read_le<uint32_t>(b + 4) != 1) return "unsupported format version";
    const uint64_t n = read_le<uint64_t>(b + 8);
    const double first = read_le<double>(b + 16), last = read_le<double>(b + 24), dt = read_le<double>(b + 32);
    if (n == 0) return "no samples";
    if (!(std::isfinite(first) && std::isfinite(last) && std::isfinite(dt) && dt > 0.0))
        return "JD start, end and step must be finite with a positive step";
    const double grid_end = first + (double)(n - 1) * dt;
    if (grid_end != last) return "declared last JD disagrees with the sample grid";
    if (b[40] != body) return "body id does not match";
    if (b[41] > 4) return "unknown epoch-scale tag";
    if (b[42] > 2) return "unknown epoch-representation tag";
    for (int i = 43; i < kHeader; ++i)
        if (b[i] != 0) return "reserved header bytes must be zero";
    if ((uint64_t)(len - kHeader) / 24 != n || (uint64_t)(len - kHeader) % 24 != 0)
        return "payload size does not match the sample count";
    Ephemeris e;
    e.pos.resize((size_t)n * 3);
    std::memcpy(e.pos.data(), b + kHeader, (size_t)n * 24);
    for (double v : e.pos)
        if (!std::isfinite(v)) return "non-finite position";
    e.n = (int64_t)n;
    e.jd_start = first;
    e.jd_end = grid_end;
    e.dt = dt;
    e.inv_dt = 1.0 / dt;
    *out = std::move(e);
    return "";
}

// For p(s) = b + s d on one piece, the unit vector turns at |b x d| / |p(s)|^2
// per grid step; the largest value is at the point of the piece closest to
// the origin.
double ephemeris_direction_rate(const Ephemeris& e) {
    if (e.n < 2 || !(std::isfinite(e.dt) && e.dt > 0.0)) return 0.0;
    double sup = 0.0;
    for (int64_t i = 0; i + 1 < e.n; ++i) {
        const double* b = &e.pos[3 * i];
        const double* a = &e.pos[3 * (i + 1)];
        const double d[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
        const double c[3] = {b[1] * d[2] - b[2] * d[1], b[2] * d[0] - b[0] * d[2], b[0] * d[1] - b[1] * d[0]};
        const double cn = std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
        const double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        const double pr = std::fma(b[0], d[0], std::fma(b[1], d[1], b[2] * d[2]));
        const double s = d2 > 0.0 ? std::min(std::max(-pr / d2, 0.0), 1.0) : 0.0;
        const double q[3] = {std::fma(s, d[0], b[0]), std::fma(s, d[1], b[1]), std::fma(s, d[2], b[2])};
        const double q2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
        if (!(std::isfinite(q2) && q2 > 0.0)) return NAN;
        sup = std::max(sup, cn / (e.dt * q2));
    }
    return sup;
}

}  // namespace bqp
