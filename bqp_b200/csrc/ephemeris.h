// Precomputed Sun / Moon catalogues on the host ("DUST" binary format of
// lightyear_odeint_rs/src/precomputed_ephem.rs, checked as its loader does,
// 680-830).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "physics.cuh"

namespace bqp {

struct Ephemeris {
    std::vector<double> pos;  // [n][3] Earth-centred ICRS km
    double jd_start = 0.0, jd_end = 0.0, dt = 0.0, inv_dt = 0.0;
    int64_t n = 0;

    // The catalogue over host memory (for host-side lookups).
    EphemTable host_view() const { return {pos.data(), jd_start, jd_end, dt, inv_dt, n}; }
};

// Parses a catalogue for body 0 (Sun) or 1 (Moon); "" on success, else the reason.
std::string parse_ephemeris(const uint8_t* bytes, int64_t len, int body, Ephemeris* out);

// Supremum of the catalogue direction's angular rate over its linear pieces,
// rad/day (the bound of the eclipse scans, precomputed_ephem.rs:947-1021);
// NaN when a piece passes through the origin.
double ephemeris_direction_rate(const Ephemeris& e);

}  // namespace bqp
