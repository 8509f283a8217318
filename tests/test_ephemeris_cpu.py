"""Precomputed Sun / Moon catalogues ("DUST" format of
lightyear_odeint_rs/src/precomputed_ephem.rs): the oracle's loader checks,
linear interpolation and endpoint rule, and the library's host pass of the
device lookup against the oracle, bit for bit."""
import os
import struct
from pathlib import Path

import numpy as np
import pytest

from bqp_b200 import _native as N
from bqp_b200 import workloads
from oracle import oracle as O

# the reference tree, when the environment names it (BQP_REFERENCE_ROOT)
REF_EPH = Path(os.environ.get("BQP_REFERENCE_ROOT", "/nonexistent")) / "dust_transfer/crates/lightyear_odeint_rs/data/ephemeris"
EPS = np.finfo(float).eps


def catalogue(pos, jd0, dt, body, scale=1, rep=1, reserved=b"\0" * 5, last=None, version=1, magic=b"DUST"):
    pos = np.ascontiguousarray(pos, dtype="<f8").reshape(-1, 3)
    n = pos.shape[0]
    if last is None:
        last = jd0 + (n - 1) * dt
    head = struct.pack("<4sIQdddBBB", magic, version, n, jd0, last, dt, body, scale, rep) + reserved
    assert len(head) == 48
    return head + pos.tobytes()


def synthetic(n=200, jd0=2460300.5, dt=0.125, seed=0, r=384400.0):
    rng = np.random.default_rng(seed)
    t = np.arange(n) * dt
    ang = 2 * np.pi * t / 27.3
    pos = np.stack([r * np.cos(ang), r * np.sin(ang) * 0.917, r * np.sin(ang) * 0.398], axis=1)
    return pos + rng.normal(0, 50.0, pos.shape), jd0, dt


def force(data=None, body="moon"):
    F = O.Force(workloads.synthetic_field(2), 2, sun=True, moon=True)
    if data is not None:
        F.set_ephemeris(body, data)
    return F


def test_grid_points_midpoints_and_ends():
    pos, jd0, dt = synthetic()
    data = catalogue(pos, jd0, dt, 1)
    F = force(data)
    n = pos.shape[0]
    jd_end = jd0 + (n - 1) * dt
    # grid points give the samples
    assert np.array_equal(F.body_positions("moon", jd0 + np.arange(n) * dt), pos)
    # midpoints: a (1 - f) + b f with f = 0.5
    mid = F.body_positions("moon", jd0 + (np.arange(n - 1) + 0.5) * dt)
    assert np.array_equal(mid, pos[:-1] * 0.5 + pos[1:] * 0.5)
    # the last JD is inside; JD roundoff past either end clamps, more is NaN
    assert np.array_equal(F.body_positions("moon", jd_end)[0], pos[-1])
    assert np.array_equal(F.body_positions("moon", jd_end + 2 * EPS * jd_end)[0], pos[-1])
    assert np.array_equal(F.body_positions("moon", jd0 - 2 * EPS * jd_end)[0], pos[0])
    for jd in (jd_end + 1e-6, jd0 - 1e-6, np.nan):
        assert np.isnan(F.body_positions("moon", jd)).all()


def test_single_sample_catalogue():
    F = force(catalogue([[1.0, 2.0, 3.0]], 2460300.5, 1.0, 0), body="sun")
    assert np.array_equal(F.body_positions("sun", 2460300.5)[0], [1.0, 2.0, 3.0])
    assert np.isnan(F.body_positions("sun", 2460300.6)).all()


def test_rejected_catalogues():
    pos, jd0, dt = synthetic(20)
    bad_pos = pos.copy()
    bad_pos[3, 1] = np.nan
    good = catalogue(pos, jd0, dt, 1)
    bad = [
        catalogue(pos, jd0, dt, 1, magic=b"DUSX"),
        catalogue(pos, jd0, dt, 1, version=2),
        catalogue(pos, jd0, -dt, 1),
        catalogue(pos, jd0, dt, 1, last=jd0 + 19 * dt + 1e-6),  # last JD off the grid
        catalogue(pos, jd0, dt, 0),  # Sun id in a Moon slot
        catalogue(pos, jd0, dt, 1, scale=5),
        catalogue(pos, jd0, dt, 1, rep=3),
        catalogue(pos, jd0, dt, 1, reserved=b"\0\0\1\0\0"),
        good[:-8],  # short payload
        catalogue(bad_pos, jd0, dt, 1),
        good[:40],
    ]
    for data in bad:
        with pytest.raises(ValueError):
            force(data)
        with pytest.raises(ValueError):
            N.ephemeris_check("moon", data)


def test_library_matches_oracle():
    pos, jd0, dt = synthetic(400, seed=3)
    data = catalogue(pos, jd0, dt, 1)
    n = pos.shape[0]
    rng = np.random.default_rng(4)
    jd_end = jd0 + (n - 1) * dt
    jds = np.concatenate([rng.uniform(jd0 - 1, jd_end + 1, 20000), jd0 + np.arange(n) * dt,
                          [jd_end, jd_end * (1 + EPS), jd0 * (1 - EPS), np.nan]])
    count, got = N.ephemeris_check("moon", data, jds)
    ref = force(data).body_positions("moon", jds)
    assert count == n
    ok = ~np.isnan(ref[:, 0])
    assert np.array_equal(np.isnan(got[:, 0]), ~ok)
    assert np.array_equal(got[ok].view(np.int64), ref[ok].view(np.int64))


@pytest.mark.skipif(not (REF_EPH / "sun.bin").exists(), reason="reference catalogues not present")
@pytest.mark.parametrize("body,n,radius", [("sun", 4019, (1.46e8, 1.53e8)), ("moon", 32145, (3.5e5, 4.1e5))])
def test_reference_catalogues(body, n, radius):
    data = (REF_EPH / f"{body}.bin").read_bytes()
    rng = np.random.default_rng(6)
    jds = rng.uniform(2458849.5, 2462867.5, 20000)
    count, got = N.ephemeris_check(body, data, jds)
    ref = force(data, body).body_positions(body, jds)
    assert count == n
    assert np.array_equal(got.view(np.int64), ref.view(np.int64))
    r = np.linalg.norm(got, axis=1)
    assert radius[0] < r.min() and r.max() < radius[1]
    # the analytic series the build uses without a catalogue stays within
    # 0.15 deg and 0.2 % in distance of it (measured: Sun 0.10 deg, 0.012 %;
    # Moon 0.09 deg, 0.14 %)
    series = force().body_positions(body, jds)
    cosang = np.sum(series * got, axis=1) / (np.linalg.norm(series, axis=1) * r)
    assert np.degrees(np.arccos(np.clip(cosang, -1, 1))).max() < 0.15
    assert (np.abs(np.linalg.norm(series, axis=1) - r) / r).max() < 2e-3
