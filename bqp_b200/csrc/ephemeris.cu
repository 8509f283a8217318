// "DUST" catalogue parsing (host code).  Layout: 48-byte little-endian header
// (4-byte magic "DUST", u32 version 1, u64 sample count, f64 first JD, f64
// last JD, f64 step in days, u8 body id, u8 epoch-scale tag 0-4, u8
// epoch-representation tag 0-2, five zero bytes), then samples x 3 f64.  The
// last JD must equal first + (samples - 1) x step as the producer rounds it,
// and every position must be finite.
#include "ephemeris.h"

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

}  // namespace bqp
