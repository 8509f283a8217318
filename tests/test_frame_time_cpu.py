"""The IAU 2006/2000A frame chain and its 1800 s segment authority, on the
host, against the reference's recorded known answers
(``tests/golden/frame_time.json``, made by ``make_frame_fixture.py``):

* ERFA's own unit-test values with ERFA's tolerances, as the reference's
  gates 2-4 hold them (satpy_core/src/frame_time/iau2006.rs, cio.rs, era.rs);
* the 20 ERFA/SOFA-derived GCRS->ITRS cases (R, Rdot, Rddot) under the
  reference's acceptance bounds (satpy_core/tests/frame_time_oracle.rs:
  686-700: 5e-13, 1e-13, 1e-12);
* the segment authority against the exact chain within the reference's
  1 mm at 7000 km (authority.rs:1405-1505), and its angular velocity
  against the fixture's Rdot at 2024-01-01 within 2e-13 rad/s
  (frame_time_oracle.rs:611-684).
"""
import json
import os
import struct
from pathlib import Path

import numpy as np
import pytest

from bqp_b200 import _native as N

GOLD = json.loads((Path(__file__).parent / "golden" / "frame_time.json").read_text())


def hx(h):
    return struct.unpack(">d", bytes.fromhex(h[2:]))[0]


def hxa(seq):
    return np.array([hx(h) for h in seq])


def test_erfa_unit_values():
    e = GOLD["erfa"]
    got = N.frame_xys06a(*e["xys06a"]["date"])
    assert np.all(np.abs(got - hxa(e["xys06a"]["want"])) < e["xys06a"]["tol"])
    for name, iau2006 in (("nut00a", False), ("nut06a", True)):
        got = N.frame_nut(*e[name]["date"], iau2006=iau2006)
        assert np.all(np.abs(got - hxa(e[name]["want"])) < e[name]["tol"]), name
    assert abs(N.frame_obl06(*e["obl06"]["date"]) - hx(e["obl06"]["want"][0])) < e["obl06"]["tol"][0]
    got = N.frame_pfw06(*e["pfw06"]["date"])
    assert np.all(np.abs(got - hxa(e["pfw06"]["want"])) < e["pfw06"]["tol"])
    c = e["c2ixys"]
    x, y, s = hxa(c["xys"])
    r = N.frame_c2ixys(x, y, s).ravel()
    assert np.all(np.abs(r[c["elements"]] - hxa(c["want"])) < c["tol"])
    assert abs(r[c["x_element"]] - x) < c["tol"]
    assert abs(N.frame_sp00(*e["sp00"]["date"]) - hx(e["sp00"]["want"][0])) < e["sp00"]["tol"][0]
    p = e["pom00"]
    r = N.frame_pom00(*p["args"]).ravel()
    assert np.all(np.abs(r[p["elements"]] - hxa(p["want"])) < p["tol"])
    assert abs(N.frame_era(*e["era00"]["date"]) - hx(e["era00"]["want"][0])) < e["era00"]["tol"][0]


@pytest.mark.parametrize("case", GOLD["cases"], ids=[c["id"] for c in GOLD["cases"]])
def test_chain_matches_erfa_sofa_derived_cases(case):
    eop = np.array([[hx(v) for v in row] for row in case["eop"]]).reshape(-1, 5)
    r, rd, rdd = N.frame_derivatives(case["epoch"], case["policy"], GOLD["stencil_h_s"], eop,
                                     case["eop_first_mjd"])
    assert np.abs(r.ravel() - hxa(case["R"])).max() <= 5e-13
    assert np.abs(rd.ravel() - hxa(case["Rdot"])).max() <= 1e-13
    assert np.abs(rdd.ravel() - hxa(case["Rddot"])).max() <= 1e-12
    # the rotation is orthonormal to rounding
    assert np.abs(r @ r.T - np.eye(3)).max() < 1e-15


def test_sealed_records_equal_the_finals_rows():
    for a in GOLD["authority"]:
        assert np.array_equal(hxa(np.ravel(a["sealed"])), hxa(np.ravel(a["finals"])))


@pytest.mark.parametrize("entry", GOLD["authority"], ids=lambda a: "%04d-%02d-%02dT%02d:%02d:%02.0f" % tuple(a["epoch"]))
def test_segments_track_the_exact_chain(entry):
    y, m, d, hh, mi, ss = entry["epoch"]
    sealed = hxa(np.ravel(entry["sealed"])).reshape(-1, 5)
    auth = N.FrameAuthority(sealed, entry["first_mjd"])
    u1, u2 = N.utc_calendar(y, m, d, hh, mi, ss)
    tai = N.tai_seconds(u1, u2)
    r, w = auth.rotation(tai)
    exact = N.frame_matrix(entry["epoch"], 1, 0.0, sealed, entry["first_mjd"])
    worst_m = 0.0
    for p in ([7000.0, 0, 0], [0, 7000.0, 0], [0, 0, 7000.0], [4041.45, 4041.45, 4041.45]):
        worst_m = max(worst_m, np.linalg.norm(r[0] @ p - exact @ p) * 1000.0)
    assert worst_m <= 1.0e-3
    # the Earth turns at about 7.292e-5 rad/s about the CIP
    assert abs(np.linalg.norm(w[0]) - 7.2921e-5) < 2e-9


def test_angular_velocity_matches_the_fixture_rate():
    case = next(c for c in GOLD["cases"] if c["id"] == "2024-01-01T00:00:00_real_eop_state_0")
    r = hxa(case["R"]).reshape(3, 3)
    rd = hxa(case["Rdot"]).reshape(3, 3)
    # passive GCRS->ITRS: R^T Rdot = -[w_gcrs x]
    m = r.T @ rd
    want = 0.5 * np.array([m[1, 2] - m[2, 1], m[2, 0] - m[0, 2], m[0, 1] - m[1, 0]])
    entry = next(a for a in GOLD["authority"] if a["epoch"][:3] == [2024, 1, 1])
    auth = N.FrameAuthority(hxa(np.ravel(entry["sealed"])).reshape(-1, 5), entry["first_mjd"])
    _, w = auth.rotation(N.tai_seconds(*N.utc_calendar(2024, 1, 1)))
    assert np.abs(w[0] - want).max() <= 2.0e-13


def test_tai_seconds_through_a_leap_second():
    # 2016-12-31 ends in a leap second: 23:59:60 is one SI second after
    # 23:59:59 and one before 2017-01-01T00:00:00 (authority.rs:1213-1247)
    t59 = N.tai_seconds(*N.utc_calendar(2016, 12, 31, 23, 59, 59.0))[0]
    t60 = N.tai_seconds(*N.utc_calendar(2016, 12, 31, 23, 59, 60.0))[0]
    t00 = N.tai_seconds(*N.utc_calendar(2017, 1, 1, 0, 0, 0.0))[0]
    assert t60 - t59 == 1.0 and t00 - t60 == 1.0
    noon = N.tai_seconds(*N.utc_calendar(2016, 12, 31, 12, 0, 0.0))[0]
    midnight = N.tai_seconds(*N.utc_calendar(2016, 12, 31, 0, 0, 0.0))[0]
    assert noon - midnight == 43200.0
    # the origin: 0h TAI of MJD 41684 is UTC 1973-01-02T00:00:00 less 12 s
    assert N.tai_seconds(*N.utc_calendar(1973, 1, 2))[0] == 12.0
    assert np.isnan(N.tai_seconds(2400000.5 + 41000.0))[0]  # 1971: before the integer-leap era


def test_segment_index_absorbs_the_interval_remainder():
    auth = N.FrameAuthority()
    iv = auth.intervals()
    # 2017-01-01 starts an interval (TAI - UTC 37 s)
    j = int(np.searchsorted(iv["start"], N.tai_seconds(*N.utc_calendar(2017, 1, 1)))[0])
    assert iv["delta_at"][j] == 37.0
    # the last instant before it belongs to the previous interval's last
    # whole segment, which therefore runs one second long
    end = iv["start"][j]
    keys, segs = auth.segments(end - 10.0, end - 0.5)
    assert len(keys) == 1
    width = end - (segs[0, 58] - 900.0)
    assert width == 1801.0
    # segments are pure functions of (j, k): the same key twice, same bits
    k2, s2 = auth.segments(end - 10.0, end - 0.5)
    assert np.array_equal(keys, k2) and np.array_equal(segs, s2)


def test_rotation_is_continuous_across_segment_edges():
    auth = N.FrameAuthority()
    t0 = N.tai_seconds(*N.utc_calendar(2024, 3, 1))[0]
    keys, segs = auth.segments(t0, t0 + 4 * 1800.0)
    edges = segs[1:, 58] - 900.0
    eps = 1e-3
    r_lo, _ = auth.rotation(edges - eps)
    r_hi, _ = auth.rotation(edges + eps)
    # 7000 km at the seam: the two interpolants meet within a millimetre
    jump = np.abs(r_hi - r_lo).max(axis=(1, 2)) * 7000.0 * 1000.0
    drift = 7.3e-5 * 2 * eps * 7000.0 * 1000.0
    assert (jump <= drift + 1e-3).all()


def test_out_of_span_instants_are_nan():
    auth = N.FrameAuthority()
    iv = auth.intervals()
    r, w = auth.rotation([iv["span_end"] + 10.0, 5.0, np.nan])
    assert np.isnan(r).all() and np.isnan(w).all()
    # with a short EOP table the span ends after its last day
    first = 60300
    auth2 = N.FrameAuthority(np.zeros((10, 5)), first)
    end = auth2.intervals()["span_end"]
    assert end == (first + 10 - 41684) * 86400.0 + 37.0
    r, _ = auth2.rotation([end - 86400.0 * 5, end - 3600.0])
    assert np.isfinite(r[0]).all()
    assert np.isnan(r[1]).all()  # its four-node interpolation runs past the table


def test_oracle_restatement_of_the_lookup_matches_the_library():
    """The oracle's own segment lookup, rotation and TAI origin (its frame
    namespace) against the library's host authority on the same segments."""
    from oracle import oracle as O
    from bqp_b200 import workloads

    auth = N.FrameAuthority()
    rng = np.random.default_rng(11)
    # UTC epochs over 1973-2049 and the half day either side of three leap seconds
    jd = np.concatenate([rng.uniform(2441684.5, 2469807.0, 400),
                         2457754.5 + rng.uniform(-0.5, 0.5, 50),
                         2450630.5 + rng.uniform(-0.5, 0.5, 50),
                         2441499.5 + rng.uniform(-0.5, 0.5, 50)])
    lib_tai = N.tai_seconds(jd)
    orc_tai = np.array([O.frame_tai_origin(j) for j in jd])
    assert np.all(np.abs(lib_tai - orc_tai) <= 2e-6)
    assert np.isnan(O.frame_tai_origin(2441000.5))  # 1971
    # rotations at instants inside one table of segments
    t0 = N.tai_seconds(2460310.5)[0]
    keys, segs = auth.segments(t0, t0 + 3 * 86400.0)
    F = O.Force(workloads.synthetic_field(2), 2)
    F.set_frame(keys, segs, auth.intervals()["raw"])
    tai = t0 + rng.uniform(0.0, 3 * 86400.0, 500)
    r_lib, w_lib = auth.rotation(tai)
    r_orc, w_orc = F.frame_rotation(tai)
    assert np.array_equal(r_lib, r_orc) and np.array_equal(w_lib, w_orc)
    # outside the segments it was given the oracle has none
    r_out, _ = F.frame_rotation([t0 - 7200.0, t0 + 4 * 86400.0])
    assert np.isnan(r_out).all()


def test_python_frame_arguments():
    """frame= / eop= of the Python calls, parsed without a GPU."""
    from bqp_b200 import api

    api._ZERO_EOP_WARNED = False
    with pytest.warns(UserWarning, match="zero EOP"):
        assert api._frame("iau2006", None)[0] == "iau2006"
    import warnings

    with warnings.catch_warnings():
        warnings.simplefilter("error")  # once per process
        assert api._frame("iau2006", None)[1] is None
    assert api._frame("gmst", None)[1] is None
    rec = np.arange(20.0).reshape(4, 5)
    name, got, first = api._frame("iau2006", (rec, 60300))
    assert np.array_equal(got, rec) and first == 60300
    # the sealed layout: 40-byte records from MJD 41684, passed as bytes
    name, got, first = api._frame("iau2006", rec.astype("<f8").tobytes())
    assert np.array_equal(got, rec) and first == 41684
    with pytest.raises(ValueError):
        api._frame("iau2006", b"\0" * 41)  # not whole records
    # IERS finals2000A text (the reference's own lines) is read as such
    entry = GOLD["authority"][0]
    name, got, first = api._frame("iau2006", ("\n".join(entry["finals_lines"]) + "\n").encode())
    assert first == entry["first_mjd"] and np.array_equal(got, hxa(np.ravel(entry["sealed"])).reshape(-1, 5))
    name, got2, _ = api._frame("iau2006", "\n".join(entry["finals_lines"]) + "\n")  # as str
    assert np.array_equal(got2, got)
    with pytest.raises(ValueError):
        api._frame("iau2006", b"no finals rows here\n")
    with pytest.raises(ValueError):
        api._frame("gmst", (rec, 60300))  # EOP belong to the IAU frame
    with pytest.raises(ValueError):
        api._frame("itrf93", None)


def test_device_segment_lookup_on_the_host(tmp_path):
    """The kernels' segment lookup (segment_index + segment_slot of
    frame_time.h, host-compiled here) on key tables with one span (the
    offset fast path), with gaps and across a leap interval (the binary
    search), against the library authority's own (j, k) keys."""
    import subprocess

    csrc = Path(__file__).resolve().parents[1] / "bqp_b200" / "csrc"
    src = tmp_path / "lookup.cpp"
    src.write_text(r'''
#include <cstdio>
#include <vector>
#include "frame_time.h"
using namespace bqp::ft;
int main() {
    // three intervals 1000 s, 5000 s and 1e9 s long from t = 12
    FrameIntervals I{};
    I.n = 3;
    I.start[0] = 12.0; I.start[1] = 1012.0; I.start[2] = 6013.0;
    I.span_end = 1e9;
    // keys: interval 0 (k 0), interval 1 (k 0, 1), interval 2 (k 0..3, 7, 8)
    std::vector<long long> k = {seg_key(0, 0), seg_key(1, 0), seg_key(1, 1), seg_key(2, 0), seg_key(2, 1),
                                seg_key(2, 2), seg_key(2, 3), seg_key(2, 7), seg_key(2, 8)};
    std::vector<int64_t> keys(k.begin(), k.end());
    FrameTab T{1, (int32_t)keys.size(), nullptr, keys.data(), &I};
    const double t[] = {5.0, 12.0, 500.0, 1011.9, 1012.0, 2811.9, 2812.0, 6012.9, 6013.0, 6013.0 + 3 * 1800 + 5,
                        6013.0 + 5 * 1800, 6013.0 + 7 * 1800 + 1, 6013.0 + 8 * 1800 + 1799, 6013.0 + 9 * 1800, 2e9};
    for (double x : t) {
        int32_t j = -1;
        int64_t kk = -1;
        const bool ok = segment_index(I, x, &j, &kk);
        std::printf("%d %d %lld %d\n", ok ? 1 : 0, j, (long long)kk, segment_slot(T, x));
    }
    // one span only: every slot by the offset path
    std::vector<int64_t> one;
    for (int q = 0; q < 40; ++q) one.push_back(seg_key(2, 100 + q));
    FrameTab T1{1, 40, nullptr, one.data(), &I};
    int bad = 0;
    for (int q = 0; q < 40; ++q) bad += segment_slot(T1, 6013.0 + (100 + q) * 1800.0 + 900.0) != q;
    std::printf("%d\n", bad);
    return 0;
}
''')
    exe = tmp_path / "lookup"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", str(csrc), str(src), "-o", str(exe)], check=True)
    lines = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = [tuple(int(v) for v in ln.split()) for ln in lines[:15]]
    assert got == [
        (0, -1, -1, -1),          # before the first interval
        (1, 0, 0, 0), (1, 0, 0, 0), (1, 0, 0, 0),  # interval 0: 1000 s, one (short) segment
        (1, 1, 0, 1),             # interval 1 starts
        (1, 1, 0, 1),             # 1799.9 s in: still k 0
        (1, 1, 1, 2),             # k 1, the last: it absorbs the remainder (5000 s = 2 x 1800 + 1400)
        (1, 1, 1, 2),
        (1, 2, 0, 3),             # interval 2
        (1, 2, 3, 6),
        (1, 2, 5, -1),            # a gap in the table: no segment
        (1, 2, 7, 7),
        (1, 2, 8, 8),
        (1, 2, 9, -1),            # past the table's last key
        (0, -1, -1, -1),          # past the span
    ], got
    assert lines[15].strip() == "0"


def test_gmst_time_staircase_against_continuous_tai():
    """Why the IAU frame takes fewer steps at eps 1e-12 than the GMST frame:
    the GMST angle is read from a one-part UTC Julian day (~2.46e6), whose
    resolution is 2^-31 d = 40 us, so the Earth-fixed frame moves in steps
    of ~2.9e-9 rad; the IAU rotation reads continuous TAI seconds (2.4e-7 s
    resolution at 1.6e9 s) and moves smoothly."""
    import ctypes as C

    from oracle import oracle as O

    L = O.lib()
    L.orc_gmst.restype = C.c_double
    L.orc_gmst.argtypes = [C.c_double]
    jd0 = 2460310.5
    t = np.arange(0.0, 400e-6, 1e-6)  # 400 us in 1 us steps
    g = np.array([L.orc_gmst(jd0 + x / 86400.0) for x in t])
    jumps = np.flatnonzero(np.diff(g) != 0.0)
    assert 5 <= jumps.size <= 15  # one jump per 40 us
    step = np.max(np.abs(np.diff(g)))
    assert 2e-9 < step < 4e-9
    auth = N.FrameAuthority()
    tai0 = N.tai_seconds(jd0)[0]
    r, _ = auth.rotation(tai0 + t)
    d = np.abs(np.diff(r[:, 0, 0]))
    assert np.count_nonzero(d) > 300  # a new value almost every microsecond
    assert d.max() < 1e-9


def test_staircase_costs_steps_at_the_tightest_tolerance():
    """The same arcs (8 of the bench's LEO rows, 70x70 + JB2008 + Sun/Moon,
    one 5400 s segment, DOP853 eps 1e-12) in the oracle: the GMST frame's
    staircase makes the step controller take many more evaluations than the
    IAU frame's smooth rotation; at eps 1e-10 the two cost the same."""
    from bqp_b200 import workloads
    from oracle import oracle as O

    text = workloads.synthetic_field(70)
    states = workloads.leo_states(65536, seed=0)[::8192]
    bal = workloads.leo_ballistics(65536, seed=0)[::8192]
    equ = np.array([O.eci2equinoc(s)[0] for s in states])
    epoch = workloads.EPOCH_JD
    F = O.Force(text, 70, drag=True, sun=True, moon=True)
    auth = N.FrameAuthority()
    tai0 = N.tai_seconds(epoch)[0]
    keys, segs = auth.segments(tai0 - 1800.0, tai0 + 5400.0 + 1800.0)
    ev = {}
    for eps in (1e-12, 1e-10):
        F.set_frame()
        _, s1, _, e1 = O.propagate_final_batch(F, O.ctrl("dop853", eps=eps), equ, epoch, 5400.0, bal)
        F.set_frame(keys, segs, auth.intervals()["raw"])
        _, s2, _, e2 = O.propagate_final_batch(F, O.ctrl("dop853", eps=eps), equ, epoch, 5400.0, bal)
        assert (s1 == 0).all() and (s2 == 0).all()
        ev[eps] = (e1.sum(), e2.sum())
    assert ev[1e-12][1] < 0.8 * ev[1e-12][0], ev
    assert abs(ev[1e-10][1] - ev[1e-10][0]) < 0.05 * ev[1e-10][0], ev


def test_finals_text_reader():
    """IERS finals2000A lines -> the sealed table's records (the reference's
    own lines and values), contiguity, skipped incomplete rows, duplicates."""
    for entry in GOLD["authority"]:
        text = "\n".join(entry["finals_lines"]) + "\n"
        rec, first = N.eop_from_finals(text)
        assert first == entry["first_mjd"] and rec.shape == (10, 5)
        assert np.array_equal(rec, hxa(np.ravel(entry["sealed"])).reshape(-1, 5))
        # CRLF line ends, and a header line, read the same
        rec2, _ = N.eop_from_finals("header\r\n" + text.replace("\n", "\r\n"))
        assert np.array_equal(rec, rec2)
    lines = GOLD["authority"][0]["finals_lines"]
    # a day whose dY field is blank ends the contiguous run
    broken = list(lines)
    broken[6] = broken[6][:116] + " " * 9 + broken[6][125:]
    rec, first = N.eop_from_finals("\n".join(broken))
    assert rec.shape == (6, 5) and first == GOLD["authority"][0]["first_mjd"]
    # a bad flag is skipped the same way; a day given twice is refused
    bad = list(lines)
    bad[3] = bad[3][:16] + "X" + bad[3][17:]
    assert N.eop_from_finals("\n".join(bad))[0].shape == (3, 5)
    with pytest.raises(ValueError):
        N.eop_from_finals("\n".join(lines + lines[:1]))
    assert N.eop_from_finals("")[0].shape == (0, 5)


@pytest.mark.parametrize("case", GOLD["cases"], ids=[c["id"] for c in GOLD["cases"]])
def test_state_transform_matches_the_fixture(case):
    """GCRS position / velocity / acceleration -> ITRS through R, Rdot, Rddot
    (chain.rs transform_state) against the fixture's, under the reference's
    state bounds (frame_time_oracle.rs:686-760: 1e-8 km, 2e-11 km/s,
    3e-10 km/s^2)."""
    eop = np.array([[hx(v) for v in row] for row in case["eop"]]).reshape(-1, 5)
    r, v, a = N.frame_transform_state(case["epoch"], hxa(case["r_gcrs"]), hxa(case["v_gcrs"]), hxa(case["a_gcrs"]),
                                      case["policy"], GOLD["stencil_h_s"], eop, case["eop_first_mjd"])
    assert np.abs(r - hxa(case["r_itrs"])).max() <= 1e-8
    assert np.abs(v - hxa(case["v_itrs"])).max() <= 2e-11
    assert np.abs(a - hxa(case["a_itrs"])).max() <= 3e-10


_REF = os.environ.get("BQP_REFERENCE_ROOT", "/nonexistent")
_FINALS = Path(_REF) / "dust_transfer/assets/reference/frame_time/finals2000A.all"
_SEALED = Path(_REF) / "dust_transfer/crates/satpy_core/src/frame_time/eop_table.bin"


@pytest.mark.skipif(not (_FINALS.exists() and _SEALED.exists()), reason="reference tree not present")
def test_finals_reader_rebuilds_the_sealed_table():
    """The reference's whole finals2000A.all, read by the library, is its
    sealed eop_table.bin bit for bit (19,645 days from MJD 41684)."""
    rec, first = N.eop_from_finals(_FINALS)
    sealed = np.frombuffer(_SEALED.read_bytes(), dtype="<f8").reshape(-1, 5)
    assert first == 41684 and rec.shape == sealed.shape == (19645, 5)
    assert np.array_equal(rec, sealed)
