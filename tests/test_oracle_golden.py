"""The CPU oracle against the reference's own golden vectors.

Pins the oracle before it is trusted as the checker of the CUDA path:
* Orekit 13.1.2 DIR-R6 d/o 5 gravity (lightyear_odeint_rs/tests/gravity_orekit_oracle.rs:862-995)
* Orekit JB2008 primitive inputs -> density, 15 cases, and the Orekit JAR
  literals of jb_rs/src/jb2008.rs (rel 5e-13)
* Orekit WGS84 geodetic altitude of the JB2008 adapter fixture
"""
import json
import struct

import numpy as np
import pytest

from oracle import oracle as O


def h(s):
    return struct.unpack(">d", bytes.fromhex(s[2:]))[0]


@pytest.fixture(scope="module")
def grav(golden_dir):
    return json.loads((golden_dir / "orekit_gravity_dir_r6_d5.json").read_text())


@pytest.fixture(scope="module")
def jbfix(golden_dir):
    return json.loads((golden_dir / "orekit_jb2008.json").read_text())


def test_gravity_matches_orekit_dir_r6(grav, golden_dir):
    field = O.Force((golden_dir / "dir_r6_d15.txt").read_text(), 5)
    tol_abs, tol_rel = h(grav["absolute_tolerance_m_s2"]), h(grav["relative_tolerance"])
    assert h(grav["gm_m3_s2"]) == 398600.4415e9
    assert h(grav["reference_radius_m"]) == 6378136.46
    for case in grav["cases"]:
        pos = np.array([h(x) for x in case["position_m"]])
        acc = field.gravity_itrs(pos / 1000.0)[0] * 1000.0
        full = np.array([h(x) for x in case["full_m_s2"]])
        pm = np.array([h(x) for x in case["point_mass_m_s2"]])
        nc = np.array([h(x) for x in case["orekit_noncentral_m_s2"]])
        mu = 398600.4415e9
        point_mass = -mu * pos / np.linalg.norm(pos) ** 3
        for got, want in ((acc, full), (point_mass, pm), (acc - point_mass, nc)):
            assert np.all(np.abs(got - want) <= tol_abs + tol_rel * np.abs(want)), case["name"]


def _jb_inputs(pi):
    return [h(pi["date_mjd_fixed_utc"]), h(pi["sun_geodetic_latitude_rad_as_sunDecli"]),
            h(pi["satellite_geodetic_longitude_rad_as_satLon"]) - h(pi["sun_longitude_rad_as_sunRA"]),
            h(pi["satellite_geodetic_latitude_rad_as_satLat"]),
            h(pi["satellite_ellipsoidal_altitude_m_as_satAlt"]),
            h(pi["f10"]), h(pi["f10b"]), h(pi["s10"]), h(pi["s10b"]), h(pi["xm10"]), h(pi["xm10b"]),
            h(pi["y10"]), h(pi["y10b"]), h(pi["dstdtc"])]


def test_jb2008_matches_orekit_fixture(jbfix):
    for case in jbfix["cases"]:
        rho = O.jb2008(_jb_inputs(case["jb_primitive_inputs"]))
        want = h(case["density_kg_m3"])
        assert abs(rho - want) / want <= jbfix["relative_tolerance"], case["id"]


def test_jb2008_matches_orekit_jar_literals(jbfix):
    L = jbfix["orekit_local_input"]
    assert len(jbfix["literals"]) == 13
    for lit in jbfix["literals"]:
        inp = [lit["mjd_utc"] or L["mjd_utc"], L["sun_declination_rad"], L["hour_angle_rad"],
               L["sat_geocentric_lat_rad"], lit["altitude_km"] * 1000.0, L["f10"], L["f10b"],
               L["s10"], L["s10b"], L["m10"], L["m10b"], L["y10"], L["y10b"], L["dtc_k"]]
        rho = O.jb2008(inp)
        want = lit["density_kg_m3"]
        assert abs(rho - want) / want <= 5e-13, lit


def test_jb2008_error_codes(jbfix):
    L = jbfix["orekit_local_input"]
    base = [L["mjd_utc"], L["sun_declination_rad"], L["hour_angle_rad"], L["sat_geocentric_lat_rad"],
            400e3, L["f10"], L["f10b"], L["s10"], L["s10b"], L["m10"], L["m10b"], L["y10"], L["y10b"],
            L["dtc_k"]]
    bad = list(base); bad[0] = float("nan")
    assert O.jb2008(bad) == -1.0
    bad = list(base); bad[4] = 89e3
    assert O.jb2008(bad) == -2.0
    bad = list(base); bad[3] = 2.0
    assert O.jb2008(bad) == -3.0
    bad = list(base); bad[6] = 0.0
    assert O.jb2008(bad) == -4.0


def test_geodetic_altitude_matches_orekit(jbfix):
    for case in jbfix["cases"]:
        p = np.array([h(x) for x in case["satellite_body_m"]]) / 1000.0
        alt = O.geodetic_altitude_km(p) * 1000.0
        assert abs(alt - h(case["satellite_geodetic"]["altitude_m"])) < 1e-6, case["id"]


def test_oracle_steppers_converge_to_one_trajectory():
    """DOP853, Vern7, Vern9 and the Dormand-Prince solver at tight tolerance
    reach the same final state (20x20 + drag + Sun/Moon, 3000 s, rectified):
    the tableaus and their error estimates drive one controller correctly."""
    import numpy as np

    from bqp_b200 import _native as N
    from bqp_b200 import workloads
    from oracle import oracle as O

    order = 20
    text = workloads.synthetic_field(order)
    F = O.Force(text, order, drag=True, sun=True, moon=True)
    states = workloads.leo_states(3, seed=13)
    bal = workloads.leo_ballistics(3, seed=13)
    equ, _ = N.eci_to_equinoctial(states)
    finals = {}
    for m in ("dop853", "vern7", "vern9", "dopri5_solver"):
        d, st, steps, _ = O.propagate_final_batch(F, O.ctrl(m, eps=1e-12), equ, 2460310.5, 3000.0, bal)
        assert (st == 0).all(), m
        finals[m] = d[:, :3]
    for m, d in finals.items():
        assert np.abs(d - finals["vern9"]).max() < 1e-6, m
