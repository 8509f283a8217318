"""Solar radiation pressure with binary eclipse on the GPU (both engines),
through the C ABI, against the oracle's restatement of the reference's
eclipse coordinator (lightyear_odeint_rs/src/eclipse_coordinator.rs,
events off).

Both sides run the same legs: main legs that hold the shadow side, a replay
of each step whose Hermite path crosses the shadow cylinder with steps of at
most 10 s, an old-side proof leg, a window leg that commits the root, and a
rebase with the side flipped.  Tolerance as for the other adaptive arcs:
each row within 2 x 10 eps per step of the oracle's final position, and step
counts within 5 %."""
import numpy as np
import pytest

from bqp_b200 import _native as N
from bqp_b200 import api, workloads
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EPOCH = workloads.EPOCH_JD
ENGINES = ["pipeline", "persistent"]
FLAGS = N.FORCE_DRAG | N.FORCE_SUN | N.FORCE_MOON


def ctx_srp(text, order, method="dop853", eps=1e-10, engine="pipeline", cr=1.3, am=0.02, srp=True):
    cfg = N.default_config()
    cfg.order = order
    cfg.force_flags = FLAGS | (N.FORCE_SRP if srp else 0)
    cfg.method = N.METHODS[method]
    cfg.eps = eps
    cfg.engine = N.ENGINES[engine]
    cfg.cr = cr
    cfg.atm_model = 7
    cfg.am_ratio = am
    return N.Context(text, cfg)


def oracle_srp(text, order, cr=1.3):
    F = O.Force(text, order, drag=True, sun=True, moon=True, atm_model=7)
    F.set_srp(True, cr)
    return F


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("method", ["dop853", "vern7"])
def test_srp_final_matches_oracle(engine, method):
    order, eps, tf, n = 20, 1e-10, 4 * 3600.0, 32
    text = workloads.synthetic_field(order)
    states = workloads.leo_states(n, seed=71)
    bal = workloads.leo_ballistics(n, seed=71)
    equ, _ = N.eci_to_equinoctial(states)
    got, st, steps, evals = ctx_srp(text, order, method, eps, engine).propagate_final(states, EPOCH, tf, ballistic=bal)
    d, _, rst, rsteps, _, _ = O.propagate_srp_batch(oracle_srp(text, order), O.ctrl(method, eps=eps), equ, EPOCH,
                                                    tf, bal)
    assert (st == 0).all() and (rst == 0).all(), (st, rst)
    plain, pst, _, _ = ctx_srp(text, order, method, eps, engine, srp=False).propagate_final(states, EPOCH, tf,
                                                                                           ballistic=bal)
    assert (pst == 0).all()
    moved = 0
    for i in range(n):
        ref = O.equinoc2eci(equ[i], tf)[0] + d[i]
        bound = 2 * max(steps[i], 1) * eps * 10
        assert np.linalg.norm(got[i, :3] - ref[:3]) <= bound, (i, np.linalg.norm(got[i, :3] - ref[:3]))
        moved += np.linalg.norm(plain[i, :3] - got[i, :3]) > 100 * bound
    assert moved >= n // 2  # SRP itself is far above the agreement
    assert np.all(np.abs(steps - rsteps) <= np.maximum(3, 0.05 * rsteps)), (steps, rsteps)


@pytest.mark.parametrize("engine", ENGINES)
def test_srp_sampled_matches_oracle(engine):
    order, eps, tf, n, am = 20, 1e-10, 3 * 3600.0, 16, 0.02
    text = workloads.synthetic_field(order)
    states = workloads.leo_states(n, seed=73)
    equ, _ = N.eci_to_equinoctial(states)
    grid = np.arange(0.0, tf + 1.0, 300.0)
    out, st, steps, _ = ctx_srp(text, order, "dop853", eps, engine, am=am).propagate_sampled(
        states, EPOCH, tf, grid, deltas=True)
    _, smp, rst, rsteps, _, nw = O.propagate_srp_batch(oracle_srp(text, order), O.ctrl("dop853", eps=eps), equ,
                                                       EPOCH, tf, (am, 2.2), t_eval=grid)
    assert (st == 0).all() and (rst == 0).all() and (nw == grid.size).all()
    for i in range(n):
        err = np.linalg.norm(out[i, :, :3] - smp[i, :, :3], axis=1)
        # the final sample is a step end; interior samples are cubic Hermite
        # interpolants of the steps around them, and where the two step
        # sequences part in the last bits they differ by the interpolant's own
        # error (the bound of the other sampled arcs' interior samples)
        assert err[-1] <= 2 * max(steps[i], 1) * eps * 10, (i, err[-1])
        assert err.max() <= 2e-5, (i, err.max())
    assert np.all(np.abs(steps - rsteps) <= np.maximum(3, 0.05 * rsteps))


@pytest.mark.parametrize("engine", ENGINES)
def test_srp_envelope_and_failure_reporting(engine):
    """A state outside the coordinator's envelope (radius 6000-50000 km) ends
    with BQP_ST_ECLIPSE_ENVELOPE on both sides; rows with A/m = 0 run
    without SRP (rhs.rs:31-36)."""
    order = 8
    text = workloads.synthetic_field(order)
    far = api.kep_to_eci(np.array([60000.0, 0.01, 10.0, 0.0, 0.0, 0.0]))
    leo = workloads.leo_states(2, seed=5)
    states = np.vstack([far, leo])
    bal = np.array([[0.02, 2.2], [0.02, 2.2], [0.0, 2.2]])
    ctx = ctx_srp(text, order, engine=engine)
    got, st, _, _ = ctx.propagate_final(states, EPOCH, 1800.0, ballistic=bal)
    equ, _ = N.eci_to_equinoctial(states)
    d, _, rst, _, _, _ = O.propagate_srp_batch(oracle_srp(text, order), O.ctrl("dop853", eps=1e-10), equ, EPOCH,
                                               1800.0, bal)
    assert st[0] == N.ST_ECLIPSE_ENVELOPE and rst[0] == N.ST_ECLIPSE_ENVELOPE
    assert np.isnan(got[0]).all()
    assert st[1] == 0 and st[2] == 0 and (rst[1:] == 0).all()
    plain, _, _, _ = ctx_srp(text, order, engine=engine, srp=False).propagate_final(states[2:], EPOCH, 1800.0,
                                                                                   ballistic=bal[2:])
    assert np.abs(plain[0, :3] - got[2, :3]).max() <= 1e-9
    with pytest.raises(ValueError, match="envelope"):
        api.propagate_final(far, EPOCH, 600.0, method="dop853")
    out = api.propagate(far, EPOCH, 600.0, method="dop853")
    assert not out["completed"] and out["terminal_event"] == "eclipse_envelope" and out["times_s"].size == 0


def test_python_defaults_with_srp_match_oracle():
    """api.propagate with every reference default, SRP included (DIR-R6 at
    degree 5, JB2008 atm_model 7, Sun/Moon, SRP with cr 1.3, Vern7 at tol
    1e-8, dt_max 300 s, the IAU 2006/2000A frame with zero EOP), against the
    oracle's coordinator on a 300 s grid over three hours."""
    eci = api.kep_to_eci(np.array([6778.137, 0.001, 51.6, 30.0, 40.0, 50.0]))
    grid = np.arange(0.0, 3 * 3600.0 + 1.0, 300.0)
    out = api.propagate(eci, EPOCH, grid[-1], times_s=grid)
    assert out["completed"] and np.array_equal(out["times_s"], grid), out["terminal_event"]
    F = O.Force(api._DEFAULT_FIELD.read_text(), 5, drag=True, sun=True, moon=True, atm_model=7)
    F.set_srp(True, 1.3)
    auth = N.FrameAuthority()
    tai0 = N.tai_seconds(EPOCH)[0]
    keys, segs = auth.segments(tai0 - 1800.0, tai0 + grid[-1] + 1800.0)
    F.set_frame(keys, segs, auth.intervals()["raw"])
    equ, rc = O.eci2equinoc(eci)
    assert rc == 0
    _, smp, st, steps, _, nw = O.propagate_srp_batch(F, O.ctrl("vern7", eps=1e-8, dt_max=300.0), equ[None], EPOCH,
                                                     grid[-1], (0.01, 2.2), t_eval=grid)
    assert st[0] == 0 and nw[0] == grid.size
    ref = np.array([O.equinoc2eci(equ, t)[0] for t in grid]) + smp[0]
    err = np.linalg.norm(out["states_eci"][:, :3] - ref[:, :3], axis=1)
    assert err[-1] <= 2 * 10 * max(out["steps"], steps[0]) * 1e-8, (err[-1], out["steps"])
    assert err.max() <= 2e-5, err
    assert abs(out["steps"] - steps[0]) <= max(3, 0.05 * steps[0])
    plain = api.propagate(eci, EPOCH, grid[-1], times_s=grid, srp=False)
    assert np.linalg.norm(plain["states_eci"][-1, :3] - out["states_eci"][-1, :3]) > 100 * err[-1]
    fin = api.propagate_final(eci, EPOCH, grid[-1])
    assert np.linalg.norm(fin[:3] - out["states_eci"][-1, :3]) <= 2 * 10 * out["steps"] * 1e-8


def test_reference_smoke_sequence_with_every_default():
    """The propagation steps of dust_transfer/tests_smoke.py as written there:
    every keyword at the reference's default (srp=True, method vern7,
    atm_model 7) except where the script itself sets one."""
    epoch = 2460310.5
    kep = np.array([7178.137, 0.01, 97.4, 125.0, 210.0, 180.0])
    eci = api.kep_to_eci(kep)
    assert np.allclose(kep, api.eci_to_kep(eci), rtol=1e-6, atol=1e-6)
    out = api.propagate(eci, epoch, tof_s=600.0, gravity_order=1, drag=False, srp=False, sun=False, moon=False)
    assert out["completed"], out
    assert abs(np.linalg.norm(out["states_eci"][-1][:3]) - np.linalg.norm(eci[:3])) < 200.0
    full = api.propagate(eci, epoch, tof_s=3600.0, times_s=np.arange(600.0, 3601.0, 600.0))
    assert full["completed"] and np.isfinite(full["states_eci"]).all(), full["terminal_event"]
    assert full["states_eci"].shape == (7, 6)
    fs = api.propagate_final(eci, epoch, tof_s=3600.0)
    assert np.linalg.norm(fs[:3] - full["states_eci"][-1][:3]) < 1e-3, "final vs sampled disagree"
    with pytest.raises(ValueError):
        api.propagate_final(api.kep_to_eci([6600.0, 0.05, 30.0, 0.0, 0.0, 0.0]), epoch, 6000.0, srp=False)


def _grazing_paths(n, seed):
    """Steps of circular LEO orbits whose planes sit at every angle to the
    Sun axis, most of them close to grazing the shadow cylinder (the scans
    that bisect longest), as Hermite path rows for bqp_ecl_scan_check."""
    rng = np.random.default_rng(seed)
    rows = np.empty((n, 16))
    for k in range(n):
        r = rng.uniform(6650.0, 7300.0)
        t0 = rng.uniform(0.0, 86400.0)
        sun, _ = O.sun_moon(O.utc_jd_at(EPOCH, t0))
        u = sun / np.linalg.norm(sun)
        graze = np.arcsin(6378.137 / r)
        beta = graze + rng.normal(0.0, 0.02) if k % 2 == 0 else rng.uniform(0.0, 1.3)
        # orbit plane at angle beta to the Sun axis
        w = np.cross(u, rng.normal(size=3))
        w /= np.linalg.norm(w)
        e1 = np.cos(beta) * u + np.sin(beta) * np.cross(w, u)
        e1 /= np.linalg.norm(e1)
        e2 = w
        om = np.sqrt(398600.4415 / r ** 3)
        ph = rng.uniform(0.0, 2 * np.pi)
        h = [10.0, 60.0, 300.0][k % 3]
        def pv(t):
            a = ph + om * (t - t0)
            return (r * (np.cos(a) * e1 + np.sin(a) * e2), r * om * (-np.sin(a) * e1 + np.cos(a) * e2))
        p0, v0 = pv(t0)
        p1, v1 = pv(t0 + h)
        rows[k] = [*p0, *v0, *p1, *v1, t0, t0 + h, t0, EPOCH]
    return rows


def test_warp_scan_equals_the_serial_scan():
    """The stage-synchronous engine's warp-cooperative crossing scan and the
    persistent engine's per-thread scan return the same status, bracket and
    bound, bit for bit, on 4,096 steps of which half sit near grazing."""
    ctx = ctx_srp(workloads.synthetic_field(8), 8)
    paths = _grazing_paths(4096, seed=5)
    serial = ctx.ecl_scan(paths, warp=False)
    warp = ctx.ecl_scan(paths, warp=True)
    assert np.array_equal(serial, warp), np.flatnonzero(np.any(serial != warp, axis=1))[:10]
    found = serial[:, 1] == 1
    assert found.sum() >= 100 and (serial[found, 6] <= 1e-6).all()
    # the rest certified free of crossings, bar a few grazing steps that
    # run out of bisections as the reference's scan would
    assert (serial[~found, 0] == 0).mean() > 0.9 and set(np.unique(serial[:, 0])) <= {0.0, 14.0, 16.0}


@pytest.mark.parametrize("engine", ENGINES)
def test_srp_mixed_orbits_match_oracle(engine):
    """SRP on LEO, MEO, GEO and HEO rows (the uneven workload's orbits, every
    row with A/m > 0) over one day: long shadows at GEO, perigee passes of
    HEO rows, both engines against the oracle."""
    order, eps, tf, n = 20, 1e-10, 86400.0, 24
    text = workloads.synthetic_field(order)
    states, _, _ = workloads.mixed_states(n, seed=29)
    bal = workloads.leo_ballistics(n, seed=29)
    equ, _ = N.eci_to_equinoctial(states)
    got, st, steps, _ = ctx_srp(text, order, "dop853", eps, engine).propagate_final(states, EPOCH, tf, ballistic=bal)
    d, _, rst, rsteps, _, _ = O.propagate_srp_batch(oracle_srp(text, order), O.ctrl("dop853", eps=eps), equ, EPOCH,
                                                    tf, bal)
    assert np.array_equal(st, rst), (st, rst)
    ok = st == 0
    assert ok.sum() >= n - 2
    # over a day of ~30 shadow crossings a LEO row's along-track error grows:
    # the oracle itself moves by up to ~1e-4 km when its input moves by
    # 1e-15, so each row is held to the larger of the per-step bound and
    # twice that spread of the oracle's own result
    spread = np.zeros(n)
    for k in (1, 2, 3):
        pe = equ.copy()
        pe[:, 0] *= 1.0 + k * 1e-15
        dk, _, _, _, _, _ = O.propagate_srp_batch(oracle_srp(text, order), O.ctrl("dop853", eps=eps), pe, EPOCH, tf,
                                                  bal)
        for i in np.flatnonzero(ok):
            a = O.equinoc2eci(equ[i], tf)[0] + d[i]
            b = O.equinoc2eci(pe[i], tf)[0] + dk[i]
            spread[i] = max(spread[i], np.linalg.norm(a[:3] - b[:3]))
    for i in np.flatnonzero(ok):
        ref = O.equinoc2eci(equ[i], tf)[0] + d[i]
        bound = max(2 * max(steps[i], 1) * eps * 10, 2 * spread[i])
        assert np.linalg.norm(got[i, :3] - ref[:3]) <= bound, (i, np.linalg.norm(got[i, :3] - ref[:3]), bound)
    assert np.all(np.abs(steps[ok] - rsteps[ok]) <= np.maximum(5, 0.1 * rsteps[ok]))
