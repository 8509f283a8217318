"""The oracle's restatement of the plain-function parts of the reference's
binary-eclipse SRP (lightyear_odeint_rs/src/eclipse.rs, rhs.rs:1269-1310),
pinned by the reference's own unit tests (eclipse.rs:494-660).  The event
coordinator that sets the side per leg is not restated."""
import numpy as np

from oracle import oracle as O

R = 6378.137
SUN = [149597870.7, 0.0, 0.0]


def test_cylinder_sides():
    # eclipse.rs: compiled_shadow_authority_is_binary_cylinder_only,
    # cylinder_boundaries_and_sunward_states_are_lit
    assert O.shadow_cylinder([-7000.0, 0.0, 0.0], SUN, R)[0] == "shadow"
    for p in ([-7000.0, R, 0.0], [0.0, 0.0, 0.0], [-0.0, 0.0, 0.0], [7000.0, 0.0, 0.0]):
        assert O.shadow_cylinder(p, SUN, R)[0] == "lit", p


def test_margins():
    # eclipse.rs: sunward_outside_cylinder_margin_ignores_harmless_terminator_crossing
    outside = R + 100.0
    assert O.shadow_cylinder([-1e-12, outside, 0.0], SUN, R)[1] > 99.0
    assert O.shadow_cylinder([1e-12, outside, 0.0], SUN, R)[1] > 99.0
    side, margin = O.shadow_cylinder([1e-12, 0.0, 0.0], SUN, R)
    assert side == "lit" and margin == 1e-12  # bit-equal
    # deep in the shadow the margin is the nearer of the axial and radial distances
    side, margin = O.shadow_cylinder([-7000.0, 100.0, 0.0], SUN, R)
    assert side == "shadow" and np.isclose(margin, R - 100.0, rtol=1e-12)


def test_invalid_geometry_fails_closed():
    # eclipse.rs: invalid_geometry_fails_closed
    for sun in ([0.0, 0.0, 0.0], [np.nan, 0.0, 0.0], [np.inf, 0.0, 0.0]):
        assert O.shadow_cylinder([-7000.0, 0.0, 0.0], sun, R) is None
    assert O.shadow_cylinder([np.nan, 0.0, 0.0], SUN, R) is None
    assert O.shadow_cylinder([-7000.0, 0.0, 0.0], SUN, 0.0) is None


def test_no_crossing_certificate():
    # eclipse.rs: no_crossing_certificate_spends_one_budget_across_the_interval
    assert O.no_crossing_certified(3.0, 2.0, 4.0)
    assert not O.no_crossing_certified(1.5, 2.0, 4.0)
    assert O.no_crossing_certified(5.0, 0.0, 4.0)
    assert not O.no_crossing_certified(4.0, 0.0, 4.0)


def test_envelope():
    # eclipse.rs: part_a_eclipse_envelope_rejects_states_outside_campaign_headroom
    assert O.eclipse_envelope_ok([7000.0, 0.0, 0.0], [0.0, 19.9, 0.0])
    assert not O.eclipse_envelope_ok([7000.0, 0.0, 0.0], [0.0, 20.1, 0.0])
    assert not O.eclipse_envelope_ok([5999.0, 0.0, 0.0], [0.0, 7.5, 0.0])
    assert not O.eclipse_envelope_ok([50001.0, 0.0, 0.0], [0.0, 1.0, 0.0])


def test_srp_acceleration():
    # rhs.rs:1269-1310: p_sun Cr A/m (AU / d)^2, away from the Sun, km/s^2
    sat = np.array([7000.0, 0.0, 0.0])
    a = O.srp_accel(sat, SUN, cr=1.3, am=0.01)
    d = SUN[0] - sat[0]
    expected = 4.56e-6 * 1.3 * 0.01 * (SUN[0] / d) ** 2 * 1e-3
    assert np.isclose(-a[0], expected, rtol=1e-14) and a[1] == a[2] == 0.0
    assert np.all(O.srp_accel(sat, SUN, shadow=True) == 0.0)
    assert np.all(O.srp_accel(sat, SUN, cr=0.0) == 0.0)
    assert np.isnan(O.srp_accel([np.nan, 0.0, 0.0], SUN)).all()


# ---------------------------------------------------------------- crossing scan
# eclipse.rs:660-862: a satellite path that dips through the cylinder boundary
# and back during t in [0, 1], and a Sun axis that swings past a parked satellite.
import struct

MAX_SEP = 1.0e-6


def padded_upper_bound(value):
    bits = struct.unpack("<q", struct.pack("<d", value))[0] + 8
    return struct.unpack("<d", struct.pack("<q", bits))[0] + 1e-9


def double_crossing_state(t):
    if not np.isfinite(t):
        return None
    offset = 8.0 * (t - 0.5) * (t - 0.5) - 1.0
    return [-7000.0, R + offset, 0.0], [0.0, 16.0 * (t - 0.5), 0.0], SUN


def double_crossing_bound(old, new):
    t0, t1 = old[0], new[0]
    max_speed = 16.0 * max(abs(t0 - 0.5), abs(t1 - 0.5))
    return padded_upper_bound(max_speed * abs(t1 - t0))


def midpoint(a, b):
    return a + 0.5 * (b - a)


def test_scan_finds_the_earliest_forward_crossing():
    err, hit = O.first_crossing_in_step(0.0, 1.0, double_crossing_state, double_crossing_bound)
    assert err is None and hit["found"]
    assert (hit["old_side"], hit["new_side"]) == ("lit", "shadow")
    assert hit["t_old"] < hit["t_new"] and hit["bound"] <= MAX_SEP
    assert abs(midpoint(hit["t_old"], hit["t_new"]) - 0.1464466094) < 1e-5
    err, second = O.first_crossing_in_step(hit["t_new"], 1.0, double_crossing_state, double_crossing_bound)
    assert err is None and second["found"]
    assert (second["old_side"], second["new_side"]) == ("shadow", "lit")
    assert hit["t_new"] < second["t_old"]


def test_scan_finds_the_earliest_backward_crossing():
    err, hit = O.first_crossing_in_step(1.0, 0.0, double_crossing_state, double_crossing_bound)
    assert err is None and hit["found"]
    assert (hit["old_side"], hit["new_side"]) == ("lit", "shadow")
    assert hit["t_old"] > hit["t_new"] and hit["bound"] <= MAX_SEP
    assert abs(midpoint(hit["t_old"], hit["t_new"]) - 0.8535533906) < 1e-5
    err, second = O.first_crossing_in_step(hit["t_new"], 0.0, double_crossing_state, double_crossing_bound)
    assert err is None and (second["old_side"], second["new_side"]) == ("shadow", "lit")
    assert hit["t_new"] > second["t_old"]


def test_scan_limit_is_a_typed_failure():
    err, _ = O.first_crossing_in_step(0.0, 1.0, double_crossing_state, double_crossing_bound, max_splits=1)
    assert err == "split_limit"


def test_adjacent_same_side_pair_is_counted_both_ways():
    t0 = 1.0
    t1 = np.nextafter(t0, 2.0)
    state = lambda t: ([-7000.0, R, 0.0], [0.0, 0.0, 0.0], SUN)
    for a, b in ((t0, t1), (t1, t0)):
        err, out = O.first_crossing_in_step(a, b, state, lambda o, n: 0.5 * MAX_SEP, max_splits=0)
        assert err is None and not out["found"] and out["collapsed_pairs"] == 1
    err, _ = O.first_crossing_in_step(t0, t1, state, lambda o, n: 2.0 * MAX_SEP, max_splits=8)
    assert err == "non_progress"


def test_nonadjacent_same_side_interval_needs_the_split_budget():
    t0 = 1.0
    t2 = np.nextafter(np.nextafter(t0, 2.0), 2.0)
    err, _ = O.first_crossing_in_step(t0, t2, lambda t: ([-7000.0, R, 0.0], [0.0, 0.0, 0.0], SUN),
                                      lambda o, n: 0.5 * MAX_SEP, max_splits=0)
    assert err == "split_limit"


def test_moving_sun_axis_reveals_hidden_crossings():
    sat = [-7000.0, R + 1.0, 0.0]
    radius = float(np.sqrt(sum(c * c for c in sat)))

    def state(t):
        theta = -0.004 * t * (1.0 - t)
        return sat, [0.0, 0.0, 0.0], [SUN[0] * np.cos(theta), SUN[0] * np.sin(theta), 0.0]

    def bound(old, new):
        t0, t1 = old[0], new[0]
        speed = max(abs(0.004 * (1.0 - 2.0 * t0)), abs(0.004 * (1.0 - 2.0 * t1)))
        return padded_upper_bound(2.0 * radius * speed * abs(t1 - t0))

    err, hit = O.first_crossing_in_step(0.0, 1.0, state, bound)
    assert err is None and hit["found"]
    assert (hit["old_side"], hit["new_side"]) == ("lit", "shadow")
    assert midpoint(hit["t_old"], hit["t_new"]) < 0.5 and hit["bound"] <= MAX_SEP
