"""JB2008 drivers from SET space-weather tables on the device: the lookup the
force kernels make against the oracle's (bit for bit), and propagations that
use the tables against the oracle's (within the integrator tolerance), on
both engines.  Tables are synthetic, seeded, in the SOLFSMY / DTCFILE formats,
around the test epoch."""
import datetime

import numpy as np
import pytest

from bqp_b200 import _native as N
from bqp_b200 import workloads
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EPOCH = 2460310.5
ENGINES = ["pipeline", "persistent"]


def tables(first_jdn, days, seed=0):
    """SOLFSMY / DTCFILE texts for `days` consecutive days from Julian day
    number first_jdn.  The indices follow one activity level (a 27-day
    rotation around 150 sfu plus daily noise) with the 81-day means on its
    smooth part, as real files do; the model's semiannual term takes
    F81c - 0.70 S81c - 0.04 M81c, and independent random indices would drive
    it far outside the range the model is made for.  dTc follows a diurnal
    wave plus noise."""
    rng = np.random.default_rng(seed)
    sol = ["# F10, S10, M10, Y10 data release synthetic", "# YYYY DDD JulianDay F10 F81c S10 S81c M10 M81c Y10 Y81c Ssrc"]
    dtc = []
    phase = rng.uniform(0, 2 * np.pi)
    for k in range(days):
        jdn = first_jdn + k
        d = datetime.date.fromordinal(jdn - 1721425)
        doy = d.timetuple().tm_yday
        mean = 150.0 + 10.0 * np.sin(2 * np.pi * k / 81.0 + phase)
        level = mean + 50.0 * np.sin(2 * np.pi * k / 27.0 + phase) + rng.normal(0.0, 5.0)
        daily = [level * f + rng.normal(0.0, 3.0) for f in (1.0, 0.95, 1.05, 1.0)]  # F10, S10, M10, Y10
        means = [mean * f for f in (1.0, 0.95, 1.05, 1.0)]
        vals = [daily[0], means[0], daily[1], means[1], daily[2], means[2], daily[3], means[3]]
        sol.append(f"{d.year} {doy} {jdn} " + " ".join(f"{v:.1f}" for v in vals) + " TEST")
        hours = 40.0 + 60.0 * np.sin(2 * np.pi * (np.arange(24) / 24.0 + k / 7.0)) + rng.normal(0.0, 10.0, 24)
        dtc.append(f"DTC {d.year} {doy} " + " ".join(str(int(round(v))) for v in hours))
    return "\n".join(sol) + "\n", "\n".join(dtc) + "\n"


def ctx_for(text, order, sol, dtc, engine="pipeline", eps=1e-10):
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
    if sol is not None:
        ctx.set_jb_drivers(sol, dtc)
    return ctx


def oracle_force(text, order, sol, dtc):
    F = O.Force(text, order, drag=True, sun=True, moon=True)
    if sol is not None:
        F.set_drivers(sol, dtc)
    return F


def test_device_lookup_matches_oracle():
    sol, dtc = tables(2460300, 24, seed=1)
    text = workloads.synthetic_field(4)
    ctx = ctx_for(text, 4, sol, dtc)
    F = oracle_force(text, 4, sol, dtc)
    rng = np.random.default_rng(2)
    jds = np.concatenate([2460300 + np.arange(-1.0, 25.0, 1 / 48.0), rng.uniform(2460295, 2460330, 20000),
                          [np.nan, 2460200.0, 2460400.0]])
    out, ok = ctx.jb_lookup(jds)
    ref, ref_ok = F.jb_lookup(jds)
    assert np.array_equal(ok, ref_ok) and ok.sum() > 10000 and (~ok).sum() > 1000
    assert np.array_equal(out[ok].view(np.int64), ref[ok].view(np.int64))
    assert np.isnan(out[~ok]).all()


@pytest.mark.parametrize("engine", ENGINES)
def test_propagation_with_tables_matches_oracle(engine):
    """Two-hour arcs from 23:00 UTC: the drivers jump at midnight and dTc
    bends at every hour.  The jump is a discontinuity in the force that the
    embedded error estimate does not see, so the oracle's own error there can
    exceed steps * eps * 10; the device solution must be as close to a 1e-13
    km solution as the oracle's is (or within that floor)."""
    order = 20
    text = workloads.synthetic_field(order)
    sol, dtc = tables(2460300, 24, seed=3)
    n = 16
    states = workloads.leo_states(n, seed=41)
    bal = workloads.leo_ballistics(n, seed=41)
    equ, _ = N.eci_to_equinoctial(states)
    epoch = EPOCH - 1.0 / 24.0
    tf = 7200.0
    eps = 1e-10
    ctx = ctx_for(text, order, sol, dtc, engine, eps)
    got, st, steps, _ = ctx.propagate_final(states, epoch, tf, ballistic=bal)
    F = oracle_force(text, order, sol, dtc)
    assert (st == 0).all()

    def positions(tol):
        d, s, _, _ = O.propagate_final_batch(F, O.ctrl("dop853", eps=tol), equ, epoch, tf, bal)
        assert (s == 0).all()
        return np.array([O.equinoc2eci(equ[i], tf)[0][:3] + d[i][:3] for i in range(n)])

    ref, truth = positions(eps), positions(1e-13)
    err = np.linalg.norm(got[:, :3] - truth, axis=1)
    err_oracle = np.linalg.norm(ref - truth, axis=1)
    assert np.all(err <= 3 * np.maximum(err_oracle, np.maximum(steps, 1) * eps * 10)), (err, err_oracle)
    # the tables are in effect: the fixed drivers give a different trajectory
    fixed, st2, _, _ = ctx_for(text, order, None, None, engine, eps).propagate_final(states, epoch, tf, ballistic=bal)
    assert (st2 == 0).all()
    moved = np.linalg.norm(fixed[:, :3] - got[:, :3], axis=1)
    assert np.median(moved) > 100 * np.median(err) and moved.max() > 1e-2


@pytest.mark.parametrize("engine", ENGINES)
def test_arc_beyond_the_tables_fails_like_the_oracle(engine):
    order = 8
    text = workloads.synthetic_field(order)
    sol, dtc = tables(2460300, 13, seed=4)  # last day: JD 2460312 (covers instants up to 2460312.5)
    n = 4
    states = workloads.leo_states(n, seed=5)
    bal = workloads.leo_ballistics(n, seed=5)
    equ, _ = N.eci_to_equinoctial(states)
    tf = np.array([3600.0, 86400.0, 3 * 86400.0, 3600.0])
    epochs = np.array([EPOCH, EPOCH, EPOCH, 2460302.0])  # the last starts inside the Y10 lag
    ctx = ctx_for(text, order, sol, dtc, engine)
    got, st, _, _ = ctx.propagate_final(states, epochs, tf, ballistic=bal)
    F = oracle_force(text, order, sol, dtc)
    ref_st = np.array([O.propagate_final_batch(F, O.ctrl("dop853", eps=1e-10), equ[i:i + 1], epochs[i], tf[i],
                                               bal[i:i + 1])[1][0] for i in range(n)])
    # a NaN density poisons the state; the next gravity call rejects its radius
    assert list(ref_st) == [0, 0, N.ST_GRAVITY_RADIUS, N.ST_GRAVITY_RADIUS]
    assert np.array_equal(st, ref_st), (st, ref_st)
    assert np.isfinite(got[:2]).all() and np.isnan(got[2:]).all()


def test_clearing_the_tables_restores_the_fixed_drivers():
    order = 8
    text = workloads.synthetic_field(order)
    sol, dtc = tables(2460300, 24, seed=6)
    states = workloads.leo_states(8, seed=7)
    bal = workloads.leo_ballistics(8, seed=7)
    ctx = ctx_for(text, order, sol, dtc)
    with_tables, _, _, _ = ctx.propagate_final(states, EPOCH, 7200.0, ballistic=bal)
    ctx.set_jb_drivers(None, None)
    cleared, st, _, _ = ctx.propagate_final(states, EPOCH, 7200.0, ballistic=bal)
    fresh, st2, _, _ = ctx_for(text, order, None, None).propagate_final(states, EPOCH, 7200.0, ballistic=bal)
    assert (st == 0).all() and (st2 == 0).all()
    assert np.abs(cleared[:, :3] - fresh[:, :3]).max() < 1e-6
    assert np.abs(with_tables[:, :3] - fresh[:, :3]).max() > 1e-4
    with pytest.raises(ValueError):
        ctx.set_jb_drivers(sol.replace("TEST", "", 1), dtc)


def test_python_surface_takes_the_tables():
    """api.* with space_weather=(solfsmy, dtcfile) runs the same tables as a
    context that was given them."""
    from bqp_b200 import api

    sol, dtc = tables(2460300, 24, seed=8)
    states = workloads.leo_states(4, seed=11)
    got, st, _, _ = api.propagate_batch_final(states, EPOCH, 3600.0, gravity_order=8, gravity_field=
                                              workloads.synthetic_field(8), tol=1e-10, space_weather=(sol, dtc),
                                              frame="gmst")
    cfg_ctx = ctx_for(workloads.synthetic_field(8), 8, sol, dtc)
    assert (st == 0).all()
    ref, st2, _, _ = cfg_ctx.propagate_final(states, EPOCH, 3600.0, ballistic=np.array([0.01, 2.2]))
    assert (st2 == 0).all()
    # same tables and settings up to the batch defaults (DOP853, eps 1e-10, A/m 0.01, Cd 2.2)
    assert np.abs(got[:, :3] - ref[:, :3]).max() < 1e-5


def test_constant_tables_give_the_fixed_drivers_bits():
    """Tables holding the default fixed drivers every day (150 sfu, dTc 0 K) give the
    fixed-driver propagation bit for bit: the per-evaluation lookup feeds the
    same density call."""
    rows = ["# F10, S10, M10, Y10 data release constant"]
    dtc_rows = []
    for k in range(40):
        jdn = 2460290 + k
        d = datetime.date.fromordinal(jdn - 1721425)
        doy = d.timetuple().tm_yday
        rows.append(f"{d.year} {doy} {jdn} " + " ".join(["150.0"] * 8) + " TEST")
        dtc_rows.append(f"DTC {d.year} {doy} " + " ".join(["0"] * 24))
    sol, dtc = "\n".join(rows) + "\n", "\n".join(dtc_rows) + "\n"
    order = 20
    text = workloads.synthetic_field(order)
    states = workloads.leo_states(257, seed=71)
    bal = workloads.leo_ballistics(257, seed=71)
    for engine in ENGINES:
        fixed = ctx_for(text, order, None, None, engine)
        for i, v in enumerate((150.0,) * 8 + (0.0,)):
            assert fixed.cfg.jb_drivers[i] == v
        with_tables = ctx_for(text, order, sol, dtc, engine)
        a = fixed.propagate_final(states, EPOCH, 7200.0, ballistic=bal)
        b = with_tables.propagate_final(states, EPOCH, 7200.0, ballistic=bal)
        assert (a[1] == 0).all() and (b[1] == 0).all()
        assert np.array_equal(a[0].view(np.int64), b[0].view(np.int64)), engine
