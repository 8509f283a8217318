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
