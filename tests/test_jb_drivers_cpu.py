"""JB2008 space-weather drivers (SOLFSMY / DTCFILE): the oracle's parsing and
lookup against the reference's known answers (jb_rs/tests/jb2008_drivers.rs),
and the library's parser against the oracle's.

The synthetic files follow the published SET formats: SOLFSMY rows
``YYYY DDD JD F10 F81c S10 S81c M10 M81c Y10 Y81c Ssrc`` after a release header,
DTCFILE rows ``DTC YYYY DDD`` plus 24 hourly dTc values (K).  Lookups apply the
JB2008 lags (F10/S10 1 day, M10 2, Y10 5) and interpolate dTc hourly with the
SET rounding.
"""
import os
from pathlib import Path

import numpy as np
import pytest

from bqp_b200 import _native as N
from bqp_b200 import workloads
from oracle import oracle as O

INT32_MIN, INT32_MAX = -(2 ** 31), 2 ** 31 - 1
# the reference tree, when the environment names it (BQP_REFERENCE_ROOT)
REF_DATA = Path(os.environ.get("BQP_REFERENCE_ROOT", "/nonexistent")) / "dust_transfer/crates/jb_rs/data/jb2008"


def solfsmy(days, year=2022, doy0=310, jd0=2459890, values=None, header="synthetic"):
    lines = [f"# F10, S10, M10, Y10 data release {header}",
             "# YYYY DDD JulianDay F10 F81c S10 S81c M10 M81c Y10 Y81c Ssrc"]
    for d in range(days):
        v = values(d) if values else [100 * (k + 1) + d for k in range(8)]
        lines.append(f"{year} {doy0 + d} {jd0 + d} " + " ".join(str(x) for x in v) + " TEST")
    return "\n".join(lines) + "\n"


def dtcfile(days, year=2022, doy0=310, value=lambda d, h: 100 * d + h):
    return "".join(f"DTC {year} {doy0 + d} " + " ".join(str(value(d, h)) for h in range(24)) + "\n"
                   for d in range(days))


def force():
    return O.Force(workloads.synthetic_field(2), 2, drag=True)


def lookup(F, jd):
    out, ok = F.jb_lookup([jd])
    return out[0], bool(ok[0])


def same_as_oracle(sol, dtc, jds):
    """The library's parser and lookup (host pass of the device code) give the
    oracle's answers bit for bit."""
    F = force()
    F.set_drivers(sol, dtc)
    ref, ref_ok = F.jb_lookup(jds)
    counts, out, ok = N.jb_drivers_check(sol, dtc, jds)
    assert counts == F.driver_counts()
    assert np.array_equal(ok, ref_ok)
    assert np.array_equal(out[ok].view(np.int64), ref[ok].view(np.int64))
    assert np.isnan(out[~ok]).all()


def test_lags_and_hourly_dtc():
    # jb2008_drivers.rs:lookup_applies_documented_lags_and_hourly_dtc_interpolation
    F = force()
    F.set_drivers(solfsmy(8), dtcfile(8))
    out, ok = lookup(F, 2459896.2708333335)  # calendar day 2459896, 18:30 UTC
    assert ok
    assert list(out) == [105.0, 205.0, 305.0, 405.0, 504.0, 604.0, 701.0, 801.0, 619.0]
    assert lookup(F, 2459894.5)[1]
    assert not lookup(F, 2459893.5)[1]  # the 5-day Y10 lag reaches before the file
    assert F.driver_counts() == (8, 8)
    same_as_oracle(solfsmy(8), dtcfile(8), [2459896.2708333335, 2459894.5, 2459893.5, 2459897.4375,
                                            2459897.4791666665, 2459999.0, float("nan")])


def test_library_matches_oracle_on_random_instants():
    rng = np.random.default_rng(3)
    sol = solfsmy(40, values=lambda d: list(np.round(rng.uniform(60, 250, 8), 1)))
    dtc = dtcfile(40, value=lambda d, h: int(rng.integers(-50, 400)))
    # whole days, half hours, hour and day boundaries, and random instants
    jds = np.concatenate([2459890 + np.arange(-1, 42, 0.5), 2459890 + np.arange(0, 41, 1 / 24.0) - 0.5,
                          rng.uniform(2459885, 2459935, 4000)])
    same_as_oracle(sol, dtc, jds)


def test_last_day_needs_next_row_only_in_hour_23():
    # jb2008_drivers.rs:final_dtc_date_needs_next_row_only_for_hour_23_interpolation
    F = force()
    F.set_drivers(solfsmy(8), dtcfile(8))
    assert lookup(F, 2459897.4375)[1]
    assert not lookup(F, 2459897.4791666665)[1]


def test_dtc_interpolation_of_extreme_values():
    # jb2008_drivers.rs:dtc_interpolation_promotes_extremes_before_subtraction
    F = force()
    ext = {(6, 18): INT32_MIN, (6, 19): INT32_MAX}
    F.set_drivers(solfsmy(8), dtcfile(8, value=lambda d, h: ext.get((d, h), 0)))
    frac = 18.5 / 24.0 - 0.0000001
    jd = 2459896.0 - 0.5 + frac
    day_jd = np.floor(jd + 0.5)
    hour = min((jd - (day_jd - 0.5) + 0.0000001) * 24.0, 23.999999999999996)
    f = hour - np.floor(hour)
    expected = np.trunc(float(INT32_MIN) + f * (float(INT32_MAX) - float(INT32_MIN)) + 0.5)
    out, ok = lookup(F, jd)
    assert ok and out[8] == expected


def test_half_hour_bias_without_day_spill():
    # jb2008_drivers.rs:set_dtcval_bias_fixes_half_hour_rounding_without_day_spill
    F = force()
    F.set_drivers(solfsmy(9, doy0=306, jd0=2459886, values=lambda d: [100] * 8),
                  dtcfile(9, doy0=306, value=lambda d, h: int(d == 7 and h == 3)))
    out, ok = lookup(F, 2459892.6041666665)
    assert ok and out[8] == 1.0
    assert lookup(F, 2459893.4999999995)[1]
    assert lookup(F, 2459893.5)[1]


def test_leap_year_rollover_parses():
    # jb2008_drivers.rs:validates_gregorian_jd_across_leap_year_rollover
    dates = [(2020, 363), (2020, 364), (2020, 365), (2020, 366), (2021, 1), (2021, 2), (2021, 3), (2021, 4)]
    sol = "# F10, S10, M10, Y10 data release rollover\n" + "".join(
        f"{y} {d} {2459212 + i} 100 200 300 400 500 600 700 800 TEST\n" for i, (y, d) in enumerate(dates))
    dtc = "".join(f"DTC {y} {d} " + " ".join(str(h) for h in range(24)) + "\n" for y, d in dates)
    F = force()
    F.set_drivers(sol, dtc)
    assert F.driver_counts() == (8, 8)


def test_rejected_files():
    # jb2008_drivers.rs:rejects_missing_nonfinite_duplicate_and_out_of_range_drivers
    sol, dtc = solfsmy(8), dtcfile(8)
    bad = [
        ("", dtc),
        (sol.replace("100 200", "NaN 200", 1), dtc),
        (sol, dtc + dtc.splitlines()[0] + "\n"),  # duplicate DTC day
        (sol, "\n".join(l for l in dtc.splitlines() if not l.startswith("DTC 2022 314 "))),  # missing day
        (sol.replace("2459892", "2459893", 1), dtc),  # date and Julian day disagree
        (sol.replace(" TEST", "", 1), dtc),  # 11 fields
        (sol.replace("# F10, S10, M10, Y10 data release", "# something else", 1), dtc),
    ]
    for s, d in bad:
        F = force()
        with pytest.raises(ValueError):
            F.set_drivers(s, d)
        with pytest.raises(ValueError):
            N.jb_drivers_check(s, d)
    F = force()
    F.set_drivers(sol, dtc)
    assert not lookup(F, 2459999.0)[1]
    assert not lookup(F, float("nan"))[1]


@pytest.mark.skipif(not (REF_DATA / "SOLFSMY.TXT").exists(), reason="reference data files not present")
def test_reference_files_known_answer():
    # jb2008_drivers.rs:approved_catalogue_oracle_over_the_compiled_data
    F = force()
    F.set_drivers((REF_DATA / "SOLFSMY.TXT").read_text(), (REF_DATA / "DTCFILE.TXT").read_text())
    out, ok = lookup(F, 2459528.0)
    assert ok
    assert tuple(out[:4]) == (88.0, 88.3, 80.2, 79.2)
    assert tuple(out[4:8]) == (102.3, 98.0, 112.3, 99.5)
    assert out[8] == 50.0
    assert F.driver_counts()[0] == 10746
    rng = np.random.default_rng(5)
    same_as_oracle((REF_DATA / "SOLFSMY.TXT").read_text(), (REF_DATA / "DTCFILE.TXT").read_text(),
                   np.concatenate([[2459528.0], rng.uniform(2445000.0, 2461200.0, 20000)]))


def test_constant_tables_reproduce_the_fixed_drivers_in_propagation():
    """A table whose every day holds the fixed drivers (150 sfu, dTc 20 K)
    gives the oracle's fixed-driver propagation bit for bit: the per-evaluation
    lookup feeds the same density call."""
    order = 8
    text = workloads.synthetic_field(order)
    import datetime

    # 40 days across the 2023 / 2024 year boundary, dated from their day numbers
    rows = ["# F10, S10, M10, Y10 data release constant"]
    dtc_rows = []
    for k in range(40):
        jdn = 2460290 + k
        d = datetime.date.fromordinal(jdn - 1721425)
        doy = d.timetuple().tm_yday
        rows.append(f"{d.year} {doy} {jdn} " + " ".join(["150.0"] * 8) + " TEST")
        dtc_rows.append(f"DTC {d.year} {doy} " + " ".join(["20"] * 24))
    sol, dtc = "\n".join(rows) + "\n", "\n".join(dtc_rows) + "\n"
    from bqp_b200 import _native as N

    states = workloads.leo_states(4, seed=3)
    bal = workloads.leo_ballistics(4, seed=3)
    equ, _ = N.eci_to_equinoctial(states)
    fixed = O.Force(text, order, drag=True, sun=True, moon=True, drivers=(150.0,) * 8 + (20.0,))
    table = O.Force(text, order, drag=True, sun=True, moon=True, drivers=(1.0,) * 8 + (0.0,))
    table.set_drivers(sol, dtc)
    ctl = O.ctrl("dop853", eps=1e-10)
    a = O.propagate_final_batch(fixed, ctl, equ, 2460310.5, 86400.0, bal)
    b = O.propagate_final_batch(table, ctl, equ, 2460310.5, 86400.0, bal)
    assert (a[1] == 0).all() and (b[1] == 0).all()
    assert np.array_equal(a[0].view(np.int64), b[0].view(np.int64))
    assert np.array_equal(a[2], b[2])
