"""The UTC / TAI seam: the propagator integrates in continuous SI seconds and
takes the JB2008 drivers, the ephemeris catalogues and the Earth's rotation
at UTC (lightyear_odeint_rs/src/rhs.rs:3090-3110, 3264-3300).  The library's
function (the one the kernels run, evaluated on the host) against the
oracle's independent restatement, and against the known answers of the
2016-12-31 leap second."""
import datetime

import numpy as np

from bqp_b200 import _native as N
from oracle import oracle as O

MJD0 = datetime.date(1858, 11, 17)
JD_MJD = 2400000.5


def mjd(y, m, d):
    return float((datetime.date(y, m, d) - MJD0).days)


def test_leap_table_matches_bulletin_c_dates():
    # the days on which TAI - UTC changed (IERS Bulletin C), 1972-2017; the
    # reference pins 32 s at 2000-01-01, 36 s at 2016-12-31 and 37 s from
    # 2017-01-01 (satpy_core/src/frame_time/timescale.rs:762-766)
    dates = [(1972, 1), (1972, 7), (1973, 1), (1974, 1), (1975, 1), (1976, 1), (1977, 1), (1978, 1), (1979, 1),
             (1980, 1), (1981, 7), (1982, 7), (1983, 7), (1985, 7), (1988, 1), (1990, 1), (1991, 1), (1992, 7),
             (1993, 7), (1994, 7), (1996, 1), (1997, 7), (1999, 1), (2006, 1), (2009, 1), (2012, 7), (2015, 7),
             (2017, 1)]
    for y, m in dates[1:]:
        day = mjd(y, m, 1) - 1.0  # the day that ends in the leap second
        # its UTC day is 86,401 s long: its last second maps to fraction 86400/86401
        jd = N.utc_jd(JD_MJD + day, 86400.0)[0]
        assert abs((jd - JD_MJD - day) - 86400.0 / 86401.0) < 1e-9, (y, m)
    # an ordinary day: 86,400 s
    assert N.utc_jd(JD_MJD + mjd(2016, 6, 1), 86400.0)[0] == JD_MJD + mjd(2016, 6, 2)


def test_2016_leap_second_known_answers():
    d = mjd(2016, 12, 31)
    e = JD_MJD + d + 86399.0 / 86401.0  # 2016-12-31T23:59:59
    got = N.utc_jd(e, np.array([0.0, 1.0, 2.0, 3.0]))
    want = [d + 86399.0 / 86401.0, d + 86400.0 / 86401.0, d + 1.0, d + 1.0 + 1.0 / 86400.0]
    assert np.all(np.abs(got - JD_MJD - np.array(want)) < 1e-9), got - JD_MJD
    # a two-day arc from 2016-12-31T00:00 across it ends one UTC second
    # before jd0 + 2 days
    start = JD_MJD + d
    assert abs((N.utc_jd(start, 2 * 86400.0)[0] - (start + 2.0)) * 86400.0 + 1.0) < 1e-4


def test_plain_where_no_leap_second_is_near():
    rng = np.random.default_rng(3)
    jd0 = JD_MJD + rng.uniform(mjd(2018, 1, 1), mjd(2030, 1, 1), 2000)
    t = rng.uniform(0.0, 30 * 86400.0, 2000)
    assert np.array_equal(N.utc_jd(jd0, t), jd0 + t / 86400.0)
    early = JD_MJD + mjd(1965, 3, 1)
    assert N.utc_jd(early, 1e5)[0] == early + 1e5 / 86400.0


def test_library_matches_oracle_around_leap_days():
    rng = np.random.default_rng(5)
    for y, m in ((2016, 12), (2015, 6), (2012, 6), (1998, 12)):
        last = mjd(y, m, 31 if m == 12 else 30)
        jd0 = JD_MJD + last + rng.uniform(-3.0, 1.5, 300)
        t = rng.uniform(0.0, 5 * 86400.0, 300)
        got = N.utc_jd(jd0, t)
        want = np.array([O.utc_jd_at(a, b) for a, b in zip(jd0, t)])
        assert np.all(np.abs(got - want) * 86400.0 < 1e-4), np.abs(got - want).max() * 86400.0
