"""The oracle's restatement of the reference's binary-eclipse coordinator
(lightyear_odeint_rs/src/eclipse_coordinator.rs, events off): its bounds
pinned by the reference's own unit tests (eclipse_coordinator.rs:3022-3120),
its trajectories checked against an independent fixed-step integration that
evaluates the shadow at every force call, and its committed roots checked on
the shadow boundary."""
import numpy as np
import pytest

from bqp_b200 import workloads as W
from oracle import oracle as O

ORDER = 8
AM, CD, CR = 0.02, 2.2, 1.3
MAX_SEP_KM = 1.0e-6          # eclipse.rs:39
MAX_ROOT_UNC_KM = 1.0e-4     # eclipse_coordinator.rs:93
SPEED_CAP = 20.0             # eclipse.rs:50


@pytest.fixture(scope="module")
def forces():
    text = W.synthetic_field(ORDER)
    plain = O.Force(text, ORDER, sun=True, moon=True)
    srp = O.Force(text, ORDER, sun=True, moon=True)
    srp.set_srp(True, CR)
    return plain, srp


def test_decisive_margin_pins():
    # post_root_decisive_margin_never_exceeds_the_detector_resolution
    err = 0.0
    for _ in range(2000):
        b, st = O.ecl_decisive_margin(err)
        assert st == 0 and 1e-9 <= b <= MAX_SEP_KM
        err += MAX_SEP_KM / 1000.0
    assert O.ecl_decisive_margin(1.0) == (MAX_SEP_KM, 0)
    assert O.ecl_decisive_margin(-1.0)[1] == 15 and O.ecl_decisive_margin(np.nan)[1] == 15
    # flat_gate_imposed_an_undeclared_transversality_floor
    window_s = MAX_ROOT_UNC_KM / SPEED_CAP
    assert 0.0906 < MAX_SEP_KM / window_s
    assert 0.0906 * window_s > 100.0 * O.ecl_decisive_margin(1.07e-12)[0]
    # post_root_skip_window_stays_far_under_the_bracket_certificate
    srp_m_s2 = 4.56e-6 * CR * AM
    assert srp_m_s2 * window_s * 43200.0 * 100.0 < MAX_SEP_KM * 1000.0


def test_replay_window_bounds(forces):
    _, F = forces
    jd = W.EPOCH_JD
    # the uncertainty is the speed cap x dt plus the diameter cap x Sun sweep
    u, st = O.ecl_replay_uncertainty(F, jd, 100.0, 100.0 + 5e-6)
    assert st == 0 and 1e-4 < u < 1.001e-4 + 2 * 50000 * F.sun_rate_bound() * 5e-6 / 86400
    # the deepest instant within 1e-4 km lies just inside 5 us, either direction
    fwd, st = O.ecl_deepest(F, jd, 100.0, 160.0, MAX_ROOT_UNC_KM)
    assert st == 0 and 4.9e-6 < fwd - 100.0 < 5e-6
    assert O.ecl_replay_uncertainty(F, jd, 100.0, fwd)[0] <= MAX_ROOT_UNC_KM
    back, st = O.ecl_deepest(F, jd, 100.0, 40.0, 2.5e-5)
    assert st == 0 and 1.2e-6 < 100.0 - back < 1.25e-6
    # a limit already within the bound is returned as is; equal instants make no progress
    assert O.ecl_deepest(F, jd, 100.0, 100.0 + 1e-7, MAX_ROOT_UNC_KM) == (100.0 + 1e-7, 0)
    assert O.ecl_deepest(F, jd, 100.0, 100.0, MAX_ROOT_UNC_KM)[1] == 14


def test_analytic_sun_rate_bound_holds(forces):
    # the constant bounds the analytic series' direction rate over a year
    _, F = forces
    jd = W.EPOCH_JD + np.arange(0.0, 366.0, 0.05)
    u = np.array([O.sun_moon(j)[0] for j in jd])
    u /= np.linalg.norm(u, axis=1)[:, None]
    ang = np.arccos(np.clip(np.sum(u[1:] * u[:-1], axis=1), -1.0, 1.0)) / 0.05
    assert ang.max() < F.sun_rate_bound() and ang.max() > 0.95 * 0.0172


def _per_call_shadow(plain, eq, jd0, tf, h=1.0):
    """RK4 on one Encke segment with the shadow side read at every force call."""
    def f(t, y):
        out = plain.rhs(eq, 0.0, jd0, AM, CD, t, y)
        b = O.equinoc2eci(eq, t)[0]
        sat = b[:3] + y[:3]
        sun, _ = O.sun_moon(O.utc_jd_at(jd0, t))
        side, _ = O.shadow_cylinder(sat, sun)
        out[3:] += O.srp_accel(sat, sun, cr=CR, am=AM, shadow=(side == "shadow"))
        return out, side

    y, t = np.zeros(6), 0.0
    sides = []
    for _ in range(int(round(tf / h))):
        k1, s = f(t, y)
        sides.append(s)
        k2, _ = f(t + h / 2, y + h / 2 * k1)
        k3, _ = f(t + h / 2, y + h / 2 * k2)
        k4, _ = f(t + h, y + h * k3)
        y = y + h / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        t += h
    return y, sum(1 for a, b in zip(sides, sides[1:]) if a != b)


def test_coordinator_matches_per_call_shadow(forces):
    plain, F = forces
    jd0, tf = W.EPOCH_JD, 3 * 3600.0
    states = W.leo_states(4, seed=3)
    ctl = O.ctrl("dop853", eps=1e-11, dt_max=300.0)
    for k in range(2):
        eq, _ = O.eci2equinoc(states[k])
        d, _, st, _, _, _ = O.propagate_srp_batch(F, ctl, eq[None], jd0, tf, (AM, CD))
        d0, st0, _, _ = O.propagate_final_batch(plain, ctl, eq[None], jd0, tf, (AM, CD))
        assert st[0] == 0 and st0[0] == 0
        y, crossings = _per_call_shadow(plain, eq, jd0, tf)
        assert crossings >= 2  # the arc passes through the shadow
        miss = np.linalg.norm(d[0, :3] - y[:3])
        effect = np.linalg.norm(d0[0, :3] - y[:3])
        assert miss < 1e-5 and effect > 100 * miss, (miss, effect)


def test_roots_sit_on_the_boundary(forces):
    _, F = forces
    jd0, tf = W.EPOCH_JD, 4 * 3600.0
    eq, _ = O.eci2equinoc(W.leo_states(4, seed=3)[0])
    ctl = O.ctrl("dop853", eps=1e-11, dt_max=300.0)
    d, roots, st, steps, evals = O.propagate_srp_roots(F, ctl, eq, jd0, tf, AM, CD)
    assert st == 0 and len(roots) >= 4 and np.all(np.diff(roots) > 0)
    # the state at each root, from the sampled output (samples leave the
    # accepted steps unchanged), is within the root budget of the boundary,
    # and the sides alternate
    t_eval = np.concatenate([[0.0], roots, [tf]])
    d2, smp, st2, _, _, nw = O.propagate_srp_batch(F, ctl, eq[None], jd0, tf, (AM, CD), t_eval=t_eval)
    assert st2[0] == 0 and nw[0] == t_eval.size
    assert np.array_equal(d2[0], d) and np.array_equal(smp[0, -1], d)
    sides = []
    for j, t in enumerate(roots):
        x = O.equinoc2eci(eq, t)[0] + smp[0, 1 + j]
        sun, _ = O.sun_moon(O.utc_jd_at(jd0, t))
        side, margin = O.shadow_cylinder(x[:3], sun)
        assert margin <= MAX_ROOT_UNC_KM, (t, margin)
        sides.append(side)
    assert all(a != b for a, b in zip(sides, sides[1:]))
