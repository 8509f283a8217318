"""CPU-side checks of the native library: it loads, exports every symbol the C
header declares, and its host-only logic (element conversions, argument and
configuration validation) behaves like the reference's.  No kernel launches."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from bqp_b200 import _native as N
from bqp_b200 import api, workloads
from oracle import oracle as O

ROOT = Path(__file__).resolve().parent.parent


def header_functions():
    text = (ROOT / "include" / "bqp_prop.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bqp_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    names = header_functions()
    assert len(names) >= 19
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(n for n, _, _ in N.SIGNATURES) == names


def test_config_struct_matches_header_layout():
    # the ctypes mirror must have the C struct's size (4*6 + 8*10 + 8*9 + 8*3 + 4*7,
    # padded to the 8-byte alignment of its doubles, + 8 for surrogate_check, + 16 for cr and p_sun)
    assert C.sizeof(N.ForceConfig) == 24 + 80 + 72 + 24 + 32 + 8 + 16
    cfg = N.default_config()
    assert cfg.order == 5 and cfg.eps == 1e-8 and cfg.dt_max == 300.0 and cfg.max_steps == 500000
    assert list(cfg.jb_drivers)[:8] == [150.0] * 8


def test_eci_equinoctial_round_trip_matches_oracle():
    states = workloads.leo_states(64, seed=3)
    equ, ok = N.eci_to_equinoctial(states)
    assert ok.all()
    for i in range(64):
        ref, rc = O.eci2equinoc(states[i])
        assert rc == 0
        assert np.allclose(equ[i], ref, rtol=1e-14, atol=1e-14)
    back = N.equinoctial_to_eci(equ, 0.0)
    assert np.allclose(back, states, rtol=0.0, atol=1e-7)  # Kepler tolerance 1e-12 rad
    # propagation on the two-body baseline
    for i in range(8):
        ref, _ = O.equinoc2eci(equ[i], 1234.5)
        got = N.equinoctial_to_eci(equ[i], 1234.5)[0]
        assert np.allclose(got, ref, rtol=1e-13, atol=1e-9)


def test_unbound_orbit_is_rejected():
    hyper = np.array([7000.0, 0.0, 0.0, 0.0, 12.0, 0.0])
    _, ok = N.eci_to_equinoctial(hyper)
    assert not ok[0]
    with pytest.raises(ValueError):
        api.propagate_final(hyper, 2460310.5, 600.0, srp=False, method="dop853")


def test_kep_round_trip_like_reference_smoke():
    # dust_transfer/tests_smoke.py:9-12
    kep = np.array([7178.137, 0.01, 97.4, 125.0, 210.0, 180.0])
    eci = api.kep_to_eci(kep)
    back = api.eci_to_kep(eci)
    assert np.allclose(kep, back, rtol=1e-6, atol=1e-6)
    with pytest.raises(ValueError):
        api.kep_to_eci([7000.0, 1.2, 0, 0, 0, 0])


def test_python_argument_validation_mirrors_binding():
    eci = api.kep_to_eci([7178.137, 0.01, 97.4, 125.0, 210.0, 180.0])
    with pytest.raises(ValueError, match="exactly 6"):
        api.propagate([1, 2, 3], 2460310.5, 600.0)
    with pytest.raises(ValueError, match="non-finite"):
        api.propagate([np.nan] * 6, 2460310.5, 600.0)
    with pytest.raises(ValueError, match="tof_s > 0"):
        api.propagate(eci, 2460310.5, -1.0, srp=False, method="dop853")
    with pytest.raises(ValueError, match="strictly increasing"):
        api.propagate(eci, 2460310.5, 600.0, times_s=[300.0, 200.0], srp=False, method="dop853")
    with pytest.raises(ValueError, match="gravity_order"):
        api.propagate(eci, 2460310.5, 600.0, gravity_order=16, srp=False, method="dop853")
    with pytest.raises(ValueError, match="unknown integrator"):
        api.propagate(eci, 2460310.5, 600.0, srp=False, method="rk4")
    with pytest.raises(ValueError, match="not built"):
        api.propagate(eci, 2460310.5, 600.0, srp=False, method="tsit5")
    with pytest.raises(ValueError, match="srp"):
        api.propagate(eci, 2460310.5, 600.0, method="dopri5")
    with pytest.raises(ValueError, match="srp"):
        api.force_config(method="dop853", rtol=1e-9, atol=1e-9)
    with pytest.raises(ValueError, match="atm_model"):
        api.propagate(eci, 2460310.5, 600.0, srp=False, method="dop853", atm_model=2)


def test_ctx_config_validation_happens_before_device_use():
    # SRP's coordinator runs with absolute control and the RK tableaus only
    cfg = N.default_config()
    cfg.force_flags |= N.FORCE_SRP
    cfg.method = N.METHODS["dopri5"]
    with pytest.raises(N.NativeError) as e:
        N.Context("2 0 -4.8e-4 0", cfg)
    assert e.value.code == N.E_UNSUPPORTED
    cfg = N.default_config()
    cfg.force_flags |= N.FORCE_SRP
    cfg.error_control = 1
    with pytest.raises(N.NativeError) as e:
        N.Context("2 0 -4.8e-4 0", cfg)
    assert e.value.code == N.E_UNSUPPORTED
    cfg = N.default_config()
    cfg.cr = -1.0
    with pytest.raises(N.NativeError) as e:
        N.Context("2 0 -4.8e-4 0", cfg)
    assert e.value.code == N.E_ARG
    cfg = N.default_config()
    cfg.order = 129
    with pytest.raises(N.NativeError) as e:
        N.Context("2 0 -4.8e-4 0", cfg)
    assert e.value.code == N.E_ARG
    cfg = N.default_config()
    cfg.eps = 0.0
    with pytest.raises(N.NativeError):
        N.Context("2 0 -4.8e-4 0", cfg)


def test_synthetic_field_rule():
    text = workloads.synthetic_field(70)
    rows = [l.split() for l in text.splitlines() if l and not l.startswith("#")]
    assert len(rows) == sum(n + 1 for n in range(2, 71))
    c20 = [float(r[2]) for r in rows if r[0] == "2" and r[1] == "0"][0]
    assert c20 == -4.84165e-4
    hi = np.array([float(r[2]) for r in rows if int(r[0]) == 70])
    assert 0.3e-5 / 4900 < hi.std() < 3e-5 / 4900
    assert all(float(r[3]) == 0.0 for r in rows if r[1] == "0")


@pytest.mark.parametrize("level", [70.0, 150.0, 250.0])
def test_jb2008_sweep_fits_self_check(level):
    """The host-built sweep fits (1-D fixed-node, 2-D altitude-dependent)
    reproduce the Boole quadrature they replace, for quiet to active drivers."""
    w = N.jb_fit_check((level,) * 8 + (20.0,))
    assert 0 <= w["fixed"] <= 4e-15
    for fam in ("mid", "uplow", "uphigh"):
        assert 0 <= w[fam] <= 1e-13, (fam, w[fam])
    lo, hi = w["tinf_range"]
    assert 300.0 < lo < hi < 3500.0


def test_tensor_core_gemm_rejects_unsupported_shapes_before_device_use():
    lib = N.lib()
    dummy = C.c_void_p(16)
    for m, n, k in [(100, 256, 64), (128, 200, 64), (128, 256, 48)]:
        rc = lib.bqp_gemm_bf16_device(m, n, k, dummy, dummy, dummy, None)
        assert rc == N.E_ARG and b"multiple" in lib.bqp_last_error()


def test_space_weather_and_ephemeris_arguments():
    """The Python surface's file arguments: shapes accepted, others rejected
    by name, without a device."""
    from bqp_b200 import api

    assert api._space_weather(None) is None
    sol, dtc, span = api._space_weather(("a", b"b"))
    assert (sol, dtc, span) == (b"a", b"b", (0.0, 0.0))
    assert api._space_weather(("a", "b", (1, 2)))[2] == (1.0, 2.0)
    with pytest.raises(ValueError, match="space_weather"):
        api._space_weather("just one file")
    assert api._ephemeris(None) == {}
    assert api._ephemeris((b"s", None)) == {"sun": b"s"}
    assert api._ephemeris({"moon": b"m"}) == {"moon": b"m"}
    with pytest.raises(ValueError, match="ephemeris"):
        api._ephemeris((b"s",))
    with pytest.raises(ValueError, match="body"):
        api._ephemeris({"mars": b"x"})


def test_workload_kep_to_eci_matches_library():
    # the workload generator's numpy conversion (no native library needed)
    # and the library's host kep_to_eci agree to rounding
    rng = np.random.default_rng(1)
    n = 1000
    kep = np.stack([rng.uniform(6700, 42000, n), rng.uniform(0, 0.8, n), rng.uniform(0, 180, n),
                    rng.uniform(0, 360, n), rng.uniform(0, 360, n), rng.uniform(0, 360, n)], 1)
    a = workloads.kep_to_eci(kep)
    b = N.kep_to_eci(kep)
    assert np.all(np.abs(a - b) <= 1e-15 * np.abs(b).max(axis=1, keepdims=True))


def test_oracle_sampled_batch_equals_rows():
    order = 8
    text = workloads.synthetic_field(order)
    F = O.Force(text, order, drag=True, sun=True, moon=True)
    states = workloads.leo_states(5, seed=2)
    bal = workloads.leo_ballistics(5, seed=2)
    equ = np.array([O.eci2equinoc(s)[0] for s in states])
    grid = np.arange(0.0, 1801.0, 60.0)
    ctl = O.ctrl("dop853", eps=1e-9)
    d, st, steps, evals, nw = O.propagate_sampled_batch(F, ctl, equ, workloads.EPOCH_JD, 1800.0, bal, grid)
    for i in range(5):
        di, si, stp, ev, nwi = O.propagate_sampled(F, ctl, equ[i], workloads.EPOCH_JD, 1800.0, bal[i, 0], bal[i, 1],
                                                   grid)
        assert si == st[i] == 0 and nwi == nw[i] == grid.size
        assert np.array_equal(di, d[i]) and stp == steps[i] and ev == evals[i]


@pytest.mark.parametrize("model", [4, 5, 6, 7])
def test_library_density_equals_oracle_bit_for_bit(model):
    # the kernels' own JB2008 function, evaluated on the host, against the
    # oracle on the reference's broad grid (models 4-7)
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from test_oracle_golden import BROAD_ALT, broad_grid_input

    rows = [broad_grid_input(mjd, alt, lat, lst) for mjd in (51999.75, 57000.25, 60648.5) for alt in BROAD_ALT
            for lat in (-75.0, 0.0, 45.0) for lst in (0.0, 12.0, 18.0)]
    got = N.jb_density(model, np.array(rows))
    want = np.array([O.jb2008_model(r, model) for r in rows])
    assert np.array_equal(got, want)
    with pytest.raises(N.NativeError):
        N.jb_density(3, np.array(rows[:1]))


@pytest.mark.parametrize("model", [5, 6, 7])
def test_fp32_density_tracks_fp64(model):
    # the split form's FP32 density against the FP64 one on the broad grid:
    # FP32 rounding (~6e-8 per operation) enters exponents of up to ~45, so
    # the density moves by ~1e-6: within 1e-5 relative up to 1000 km, where
    # drag matters, and 5e-5 above (the hydrogen term's exponent is a
    # difference of large numbers; above 2500 km the density is capped)
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from test_oracle_golden import BROAD_ALT, broad_grid_input

    rows = np.array([broad_grid_input(mjd, alt, lat, lst) for mjd in (51999.75, 57000.25, 60648.5)
                     for alt in BROAD_ALT for lat in (-75.0, 0.0, 45.0) for lst in (0.0, 12.0, 18.0)])
    f64 = N.jb_density(model, rows)
    f32 = N.jb_density(model, rows, fp32=True)
    assert (f32 > 0).all()
    rel = np.abs(f32 - f64) / f64
    low = rows[:, 4] <= 1000e3
    assert rel[low].max() <= 1e-5 and rel.max() <= 5e-5, (rel[low].max(), rel.max())
    with pytest.raises(N.NativeError):
        N.jb_density(4, rows[:1], fp32=True)
