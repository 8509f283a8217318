"""Precomputed Sun / Moon catalogues on the device: the positions the force
kernels take against the oracle's (bit for bit), and propagations that use
the catalogues against the oracle's, on both engines.  The catalogues are
built here in the "DUST" format by sampling the analytic series on the
reference catalogues' grids (Sun daily, Moon every 3 hours)."""
import struct

import numpy as np
import pytest

from bqp_b200 import _native as N
from bqp_b200 import workloads
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EPOCH = 2460310.5
ENGINES = ["pipeline", "persistent"]


def catalogue(body, jd0, days, dt):
    F = O.Force(workloads.synthetic_field(2), 2, sun=True, moon=True)
    n = int(round(days / dt)) + 1
    pos = F.body_positions(body, jd0 + np.arange(n) * dt)
    head = struct.pack("<4sIQdddBBB5x", b"DUST", 1, n, jd0, jd0 + (n - 1) * dt, dt, N.BODIES[body], 1, 1)
    return head + np.ascontiguousarray(pos, dtype="<f8").tobytes()


def catalogues(jd0=2460300.5, days=20):
    return catalogue("sun", jd0, days, 1.0), catalogue("moon", jd0, days, 0.125)


def ctx_for(text, order, cats, engine="pipeline", eps=1e-10):
    cfg = N.default_config()
    cfg.order = order
    cfg.force_flags = N.FORCE_DRAG | N.FORCE_SUN | N.FORCE_MOON
    cfg.atm_model = 4
    cfg.method = N.METHODS["dop853"]
    cfg.error_control = 0
    cfg.eps = eps
    cfg.dt_max = 300.0
    cfg.engine = N.ENGINES[engine]
    cfg.max_kernel_seconds = 120.0
    ctx = N.Context(text, cfg)
    if cats:
        ctx.set_ephemeris("sun", cats[0])
        ctx.set_ephemeris("moon", cats[1])
    return ctx


def oracle_force(text, order, cats):
    F = O.Force(text, order, drag=True, sun=True, moon=True)
    if cats:
        F.set_ephemeris("sun", cats[0])
        F.set_ephemeris("moon", cats[1])
    return F


def test_device_positions_match_oracle():
    cats = catalogues()
    text = workloads.synthetic_field(4)
    ctx = ctx_for(text, 4, cats)
    F = oracle_force(text, 4, cats)
    rng = np.random.default_rng(1)
    jd_end = 2460320.5
    jds = np.concatenate([rng.uniform(2460299.0, 2460322.0, 20000), 2460300.5 + np.arange(161) * 0.125,
                          [jd_end * (1 + np.finfo(float).eps), np.nan]])
    for body in ("sun", "moon"):
        got = ctx.body_positions(body, jds)
        ref = F.body_positions(body, jds)
        ok = ~np.isnan(ref[:, 0])
        assert ok.sum() > 15000 and (~ok).sum() > 1000
        assert np.array_equal(np.isnan(got[:, 0]), ~ok)
        assert np.array_equal(got[ok].view(np.int64), ref[ok].view(np.int64))
    # without a catalogue the analytic series apply, as in the oracle (to the
    # last bits: the device series contracts into FMAs, the oracle does not)
    plain = ctx_for(text, 4, None)
    for body in ("sun", "moon"):
        got = plain.body_positions(body, jds[:1000])
        ref = oracle_force(text, 4, None).body_positions(body, jds[:1000])
        assert np.all(np.linalg.norm(got - ref, axis=1) <= 1e-12 * np.linalg.norm(ref, axis=1))


@pytest.mark.parametrize("engine", ENGINES)
def test_propagation_with_catalogues_matches_oracle(engine):
    order = 20
    text = workloads.synthetic_field(order)
    cats = catalogues()
    n = 16
    states = workloads.leo_states(n, seed=43)
    bal = workloads.leo_ballistics(n, seed=43)
    equ, _ = N.eci_to_equinoctial(states)
    tf = 8000.0
    eps = 1e-10
    got, st, steps, _ = ctx_for(text, order, cats, engine, eps).propagate_final(states, EPOCH, tf, ballistic=bal)
    assert (st == 0).all()
    F = oracle_force(text, order, cats)

    def positions(tol):
        d, s, _, _ = O.propagate_final_batch(F, O.ctrl("dop853", eps=tol), equ, EPOCH, tf, bal)
        assert (s == 0).all()
        return np.array([O.equinoc2eci(equ[i], tf)[0][:3] + d[i][:3] for i in range(n)])

    # linear interpolation bends the forcing at every sample, which the error
    # estimate does not see: judge the device solution by how close it is to a
    # 1e-13 km solution next to the oracle's own distance (or the step floor)
    ref, truth = positions(eps), positions(1e-13)
    err = np.linalg.norm(got[:, :3] - truth, axis=1)
    err_oracle = np.linalg.norm(ref - truth, axis=1)
    assert np.all(err <= 3 * np.maximum(err_oracle, np.maximum(steps, 1) * eps * 10)), (err, err_oracle)


@pytest.mark.parametrize("engine", ENGINES)
def test_arc_beyond_the_catalogue_fails_like_the_oracle(engine):
    order = 8
    text = workloads.synthetic_field(order)
    cats = catalogues(2460300.5, 11)  # both end at JD 2460311.5
    n = 3
    states = workloads.leo_states(n, seed=9)
    bal = workloads.leo_ballistics(n, seed=9)
    equ, _ = N.eci_to_equinoctial(states)
    tf = np.array([3600.0, 2 * 86400.0, 3600.0])
    epochs = np.array([EPOCH, EPOCH, 2460299.0])
    got, st, _, _ = ctx_for(text, order, cats, engine).propagate_final(states, epochs, tf, ballistic=bal)
    F = oracle_force(text, order, cats)
    ref_st = np.array([O.propagate_final_batch(F, O.ctrl("dop853", eps=1e-10), equ[i:i + 1], epochs[i], tf[i],
                                               bal[i:i + 1])[1][0] for i in range(n)])
    assert list(ref_st) == [0, N.ST_GRAVITY_RADIUS, N.ST_GRAVITY_RADIUS]
    assert np.array_equal(st, ref_st), (st, ref_st)
    assert np.isfinite(got[0]).all() and np.isnan(got[1:]).all()


def test_python_surface_takes_the_catalogues():
    from bqp_b200 import api

    cats = catalogues()
    states = workloads.leo_states(4, seed=12)
    text = workloads.synthetic_field(8)
    got, st, _, _ = api.propagate_batch_final(states, EPOCH, 3600.0, gravity_order=8, gravity_field=text,
                                              tol=1e-10, ephemeris=cats, frame="gmst")
    ref, st2, _, _ = ctx_for(text, 8, cats).propagate_final(states, EPOCH, 3600.0, ballistic=np.array([0.01, 2.2]))
    assert (st == 0).all() and (st2 == 0).all()
    assert np.abs(got[:, :3] - ref[:, :3]).max() < 1e-5


@pytest.mark.parametrize("engine", ENGINES)
def test_srp_with_catalogues_matches_oracle(engine):
    """Binary-eclipse SRP with the Sun from a catalogue: the shadow geometry,
    the eclipse scans and their Sun-sweep bound (the catalogue's own rate
    supremum) on both sides."""
    order, eps, tf, n = 12, 1e-10, 3 * 3600.0, 16
    text = workloads.synthetic_field(order)
    cats = catalogues()
    ctx = ctx_for(text, order, cats, engine, eps)
    cfg = N.default_config()
    cfg.order = order
    cfg.force_flags = N.FORCE_DRAG | N.FORCE_SUN | N.FORCE_MOON | N.FORCE_SRP
    cfg.atm_model = 4
    cfg.method = N.METHODS["dop853"]
    cfg.eps = eps
    cfg.engine = N.ENGINES[engine]
    cfg.cr = 1.3
    ctx.set_config(cfg)
    states = workloads.leo_states(n, seed=17)
    bal = workloads.leo_ballistics(n, seed=17)
    equ, _ = N.eci_to_equinoctial(states)
    got, st, steps, _ = ctx.propagate_final(states, EPOCH, tf, ballistic=bal)
    F = oracle_force(text, order, cats)
    F.set_srp(True, 1.3)
    d, _, rst, rsteps, _, _ = O.propagate_srp_batch(F, O.ctrl("dop853", eps=eps), equ, EPOCH, tf, bal)
    assert (st == 0).all() and (rst == 0).all(), (st, rst)
    for i in range(n):
        ref = O.equinoc2eci(equ[i], tf)[0] + d[i]
        assert np.linalg.norm(got[i, :3] - ref[:3]) <= 2 * max(steps[i], 1) * eps * 10, i
    assert np.all(np.abs(steps - rsteps) <= np.maximum(3, 0.05 * rsteps))
    # the bound the oracle uses is the catalogue's supremum, near the Sun's
    # apparent rate and below the analytic series' constant
    assert 0.0160 < F.sun_rate_bound() < 0.0185
