"""The IAU 2006/2000A Earth-fixed frame on the device (bqp_ctx_set_frame):
force evaluations and propagations against the oracle given the same
segments, on both engines, with zero EOP and with EOP records; the frame-time
failure of an instant without a segment; and the size of the frame's effect
against the GMST rotation."""
import numpy as np
import pytest

from bqp_b200 import _native as N
from bqp_b200 import workloads
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EPOCH = workloads.EPOCH_JD  # 2024-01-01T00:00:00 UTC
ENGINES = ["pipeline", "persistent"]


def eop_records(first_mjd, n, seed=7):
    """Smooth seeded Bulletin-A-like records: polar motion ~0.1-0.4 arcsec,
    UT1-UTC ~ -0.05 s drifting 1 ms/day, nutation offsets ~0.3 mas."""
    rng = np.random.default_rng(seed)
    d = np.arange(n, dtype=np.float64)
    ph = rng.uniform(0, 2 * np.pi, 5)
    return np.stack([0.15 + 0.1 * np.sin(2 * np.pi * d / 433 + ph[0]),
                     0.35 + 0.1 * np.cos(2 * np.pi * d / 433 + ph[1]),
                     -0.05 - 0.001 * d + 0.0005 * np.sin(2 * np.pi * d / 14 + ph[2]),
                     0.3 * np.sin(2 * np.pi * d / 30 + ph[3]),
                     -0.2 * np.cos(2 * np.pi * d / 30 + ph[4])], axis=1)


def make_ctx(text, order, engine, eps=1e-10, flags=N.FORCE_DRAG | N.FORCE_SUN | N.FORCE_MOON):
    cfg = N.default_config()
    cfg.order = order
    cfg.force_flags = flags
    cfg.atm_model = 4
    cfg.method = N.METHODS["dop853"]
    cfg.error_control = 0
    cfg.eps = eps
    cfg.dt_max = 300.0
    cfg.engine = N.ENGINES[engine]
    cfg.max_kernel_seconds = 120.0
    return N.Context(text, cfg)


def oracle_with_frame(text, order, epochs, t_hi, eop=None, first_mjd=41684):
    F = O.Force(text, order, drag=True, sun=True, moon=True)
    auth = N.FrameAuthority(eop, first_mjd)
    tai0 = N.tai_seconds(np.atleast_1d(epochs))
    keys, segs = auth.segments(np.nanmin(tai0) - 1800.0, np.nanmax(tai0) + t_hi + 1800.0)
    F.set_frame(keys, segs, auth.intervals()["raw"])
    return F


def final_positions(F, equ, epochs, tf, bal, eps):
    n = equ.shape[0]
    d, s, steps, _ = O.propagate_final_batch(F, O.ctrl("dop853", eps=eps), equ, epochs, tf, bal)
    pos = np.array([O.equinoc2eci(equ[i], np.broadcast_to(tf, (n,))[i])[0][:3] + d[i][:3] for i in range(n)])
    return pos, s, steps


def test_force_evaluation_matches_oracle():
    order = 20
    text = workloads.synthetic_field(order)
    ctx = make_ctx(text, order, "pipeline")
    ctx.set_frame("iau2006")
    n = 256
    rng = np.random.default_rng(3)
    states = workloads.leo_states(n, seed=5)
    equ, _ = N.eci_to_equinoctial(states)
    epochs = EPOCH + rng.uniform(0.0, 3.0, n)
    seg_t0 = np.zeros(n)
    t = rng.uniform(0.0, 20000.0, n)
    delta = rng.normal(0.0, 0.5, (n, 6)) * [1, 1, 1, 1e-3, 1e-3, 1e-3]
    bal = workloads.leo_ballistics(n, seed=5)
    got = ctx.rhs(equ, seg_t0, epochs, t, delta, ballistic=bal)
    F = oracle_with_frame(text, order, epochs, 20000.0)
    ref = np.array([F.rhs(equ[i], 0.0, epochs[i], bal[i, 0], bal[i, 1], t[i], delta[i]) for i in range(n)])
    assert np.array_equal(got[:, :3], ref[:, :3])
    base = np.array([O.equinoc2eci(equ[i], t[i])[0][:3] for i in range(n)])
    scale = 398600.4415 / np.linalg.norm(base + delta[:, :3], axis=1) ** 2  # full-field magnitude
    assert np.all(np.abs(got[:, 3:] - ref[:, 3:]).max(axis=1) <= 1e-12 * scale)
    # the same rows in the GMST frame differ by the precession-nutation angles
    gm = make_ctx(text, order, "pipeline").rhs(equ, seg_t0, epochs, t, delta, ballistic=bal)
    dif = np.linalg.norm(gm[:, 3:] - got[:, 3:], axis=1)
    assert np.median(dif / scale) > 1e-9


@pytest.mark.parametrize("engine", ENGINES)
def test_final_states_match_oracle_zero_eop(engine):
    order, eps, n = 20, 1e-10, 24
    text = workloads.synthetic_field(order)
    states = workloads.leo_states(n, seed=43)
    bal = workloads.leo_ballistics(n, seed=43)
    equ, _ = N.eci_to_equinoctial(states)
    epochs = EPOCH + np.linspace(0.0, 2.5, n)
    tf = 6 * 3600.0
    ctx = make_ctx(text, order, engine, eps)
    ctx.set_frame("iau2006")
    got, st, steps, _ = ctx.propagate_final(states, epochs, tf, ballistic=bal)
    assert (st == 0).all()
    F = oracle_with_frame(text, order, epochs, tf)
    ref, rst, _ = final_positions(F, equ, epochs, tf, bal, eps)
    assert (rst == 0).all()
    err = np.linalg.norm(got[:, :3] - ref, axis=1)
    assert np.all(err <= np.maximum(1e-6, 10 * eps * steps)), err
    # against the GMST frame the trajectories part by far more than that
    gm, gst, _, _ = make_ctx(text, order, engine, eps).propagate_final(states, epochs, tf, ballistic=bal)
    assert (gst == 0).all()
    assert np.median(np.linalg.norm(gm[:, :3] - got[:, :3], axis=1)) > 1e-3


@pytest.mark.parametrize("engine", ENGINES)
def test_sampled_states_match_oracle_with_eop(engine):
    order, eps, n = 12, 1e-10, 12
    text = workloads.synthetic_field(order)
    first = 60300  # 2023-12-22
    eop = eop_records(first, 30)
    states = workloads.leo_states(n, seed=17)
    equ, _ = N.eci_to_equinoctial(states)
    tf = 4 * 3600.0
    t_eval = np.linspace(0.0, tf, 9)
    ctx = make_ctx(text, order, engine, eps)
    ctx.set_frame("iau2006", eop, first)
    out, st, steps, _ = ctx.propagate_sampled(states, EPOCH, tf, t_eval)
    assert (st == 0).all()
    cfg = N.default_config()
    bal = np.array([cfg.am_ratio, cfg.cd])  # the context's ballistics
    F = oracle_with_frame(text, order, [EPOCH], tf, eop, first)
    d, rst, _, _, _ = O.propagate_sampled_batch(F, O.ctrl("dop853", eps=eps), equ, EPOCH, tf, bal, t_eval)
    assert (rst == 0).all()
    for i in range(n):
        ref = np.array([O.equinoc2eci(equ[i], tk)[0][:3] + d[i, k, :3] for k, tk in enumerate(t_eval)])
        err = np.linalg.norm(out[i, :, :3] - ref, axis=1)
        assert np.all(err <= max(2e-5, 10 * eps * steps[i])), (i, err)
    # the records matter: zero EOP moves the answer by metres
    z = make_ctx(text, order, engine, eps)
    z.set_frame("iau2006")
    oz, _, _, _ = z.propagate_sampled(states, EPOCH, tf, t_eval)
    assert np.median(np.linalg.norm(oz[:, -1, :3] - out[:, -1, :3], axis=1)) > 1e-4


@pytest.mark.parametrize("engine", ENGINES)
def test_instants_without_a_segment_fail_like_the_oracle(engine):
    order, eps = 8, 1e-10
    text = workloads.synthetic_field(order)
    first = 60300
    eop = eop_records(first, 14)  # through MJD 60313 (2024-01-04)
    states = workloads.leo_states(3, seed=9)
    bal = workloads.leo_ballistics(3, seed=9)
    equ, _ = N.eci_to_equinoctial(states)
    # row 0 inside the table; row 1 runs past its end; row 2 starts in 1969
    epochs = np.array([EPOCH, EPOCH + 1.5, 2440300.5])
    tf = np.array([3600.0, 2 * 86400.0, 3600.0])
    ctx = make_ctx(text, order, engine, eps)
    ctx.set_frame("iau2006", eop, first)
    got, st, _, _ = ctx.propagate_final(states, epochs, tf, ballistic=bal)
    F = oracle_with_frame(text, order, epochs[:2], 2 * 86400.0, eop, first)
    ref_st = np.array([O.propagate_final_batch(F, O.ctrl("dop853", eps=eps), equ[i:i + 1], epochs[i], tf[i],
                                               bal[i:i + 1])[1][0] for i in range(3)])
    assert list(ref_st) == [0, N.ST_FRAME_TIME, N.ST_FRAME_TIME]
    assert np.array_equal(st, ref_st), (st, ref_st)
    assert np.isfinite(got[0]).all() and np.isnan(got[1:]).all()


def test_python_surface_takes_the_frame():
    from bqp_b200 import api

    text = workloads.synthetic_field(8)
    state = workloads.leo_states(1, seed=21)[0]
    first = 60300
    eop = eop_records(first, 30)
    r_iau = api.propagate_final(state, EPOCH, 3600.0, gravity_order=8, gravity_field=text, srp=False,
                                frame="iau2006", eop=(eop, first))
    r_gm = api.propagate_final(state, EPOCH, 3600.0, gravity_order=8, gravity_field=text, srp=False,
                               frame="gmst")
    assert np.linalg.norm(r_iau[:3] - r_gm[:3]) > 1e-4
    # the default frame is the IAU one (zero EOP), as in the reference
    r_def = api.propagate_final(state, EPOCH, 3600.0, gravity_order=8, gravity_field=text, srp=False)
    r_zero = api.propagate_final(state, EPOCH, 3600.0, gravity_order=8, gravity_field=text, srp=False,
                                 frame="iau2006")
    assert np.array_equal(r_def, r_zero) and np.linalg.norm(r_def[:3] - r_iau[:3]) > 0.0
    # a sealed-format byte table from MJD 41684 is accepted as is
    sealed = np.zeros((first + 40 - 41684, 5))
    sealed[first - 41684:first - 41684 + 30] = eop
    r_sealed = api.propagate_final(state, EPOCH, 3600.0, gravity_order=8, gravity_field=text, srp=False,
                                   frame="iau2006", eop=sealed.astype("<f8").tobytes())
    assert np.abs(r_sealed - r_iau).max() < 1e-9
    with pytest.raises(RuntimeError, match="frame_invalid_time"):
        api.propagate_final(state, 2440300.5, 3600.0, gravity_order=8, gravity_field=text, srp=False,
                            frame="iau2006")
    with pytest.raises(ValueError):
        api.propagate_final(state, EPOCH, 3600.0, gravity_order=8, gravity_field=text, srp=False,
                            frame="itrf")


@pytest.mark.parametrize("engine", ENGINES)
def test_preset_span_gives_the_same_bits(engine):
    """Segments built once for a span (bqp_ctx_set_frame_span) and per call
    are the same segments: the same rows give the same bits, and a second
    run of the same batch repeats them."""
    order, eps, n = 12, 1e-10, 64
    text = workloads.synthetic_field(order)
    states = workloads.leo_states(n, seed=31)
    bal = workloads.leo_ballistics(n, seed=31)
    epochs = EPOCH + np.linspace(0.0, 1.0, n)
    tf = 3 * 3600.0
    per_call = make_ctx(text, order, engine, eps)
    per_call.set_frame("iau2006")
    a = per_call.propagate_final(states, epochs, tf, ballistic=bal)
    b = per_call.propagate_final(states, epochs, tf, ballistic=bal)
    span = make_ctx(text, order, engine, eps)
    span.set_frame("iau2006")
    span.set_frame_span(EPOCH - 0.5, EPOCH + 2.0)
    c = span.propagate_final(states, epochs, tf, ballistic=bal)
    assert (a[1] == 0).all()
    for other in (b, c):
        assert np.array_equal(a[0], other[0]) and np.array_equal(a[1], other[1])
        assert np.array_equal(a[2], other[2]) and np.array_equal(a[3], other[3])
    # a row outside the preset span fails with the frame-time status
    late = span.propagate_final(states[:2], EPOCH + 3.0, tf, ballistic=bal[:2])
    assert (late[1] == N.ST_FRAME_TIME).all()
    # back to per-call segments
    span.set_frame_span(0.0, 0.0)
    late = span.propagate_final(states[:2], EPOCH + 3.0, tf, ballistic=bal[:2])
    assert (late[1] == 0).all()
