// JB2008 space-weather tables on the host: the SET SOLFSMY (daily F10, S10,
// M10, Y10 and their 81-day centred means) and DTCFILE (hourly dTc) files,
// parsed and checked as jb_rs/src/drivers.rs does (1025-1240), and the bounds
// of the exospheric temperature they can produce over a span of days.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "jb2008.cuh"

namespace bqp {

struct SpaceWeather {
    std::vector<double> solar;  // [n_solar][8]
    std::vector<int32_t> dtc;   // [n_dtc][24]
    double first_jd = 0.0;      // Julian day number of solar row 0
    int32_t n_solar = 0;
    int32_t n_dtc = 0;
    int32_t dtc_first = 0;      // solar row of DTC row 0

    // The table over host memory (for host-side lookups).
    jb::DriverTable host_view() const {
        return {solar.data(), dtc.data(), first_jd, n_solar, n_dtc, dtc_first};
    }
};

// Parses both files; "" on success, else the reason (the table is untouched).
std::string parse_space_weather(const char* solfsmy, int64_t solfsmy_len, const char* dtcfile, int64_t dtcfile_len,
                                SpaceWeather* out);

// Exospheric-temperature bounds (K) over every lookup of the UTC days
// [jd_lo, jd_hi] (jd_lo = jd_hi = 0: the whole table), margins included, for
// sizing the drag sweep fits; false when no day in the span has its lagged
// rows.
bool space_weather_tinf_range(const SpaceWeather& sw, double jd_lo, double jd_hi, double* tlo, double* thi);

}  // namespace bqp
