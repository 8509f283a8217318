"""The allocation-free entry point (bqp_propagate_final_noalloc) against the
ordinary host-buffer entry point (bqp_propagate_final) on the same kernel.

It stages through one fixed device array shared by every call, so the test
makes two calls in a row with different batches: the second must not see
anything the first left behind.  This file sorts last so that it also runs
after every other GPU test in one process."""
import numpy as np
import pytest

from bqp_b200 import _native as N
from bqp_b200 import workloads

pytestmark = pytest.mark.gpu

EPOCH = workloads.EPOCH_JD


def make_ctx(text, order):
    cfg = N.default_config()
    cfg.engine = N.ENGINES["persistent"]
    cfg.order = order
    cfg.force_flags = N.FORCE_DRAG | N.FORCE_SUN | N.FORCE_MOON
    cfg.method = N.METHODS["dop853"]
    cfg.eps = 1e-10
    return N.Context(text, cfg)


def check_same(a, b):
    out_a, st_a, steps_a, evals_a = a
    out_b, st_b, steps_b, evals_b = b
    assert (st_a == st_b).all()
    ok = st_b == 0
    # the tolerance of the engine-agreement test: 1e-6 km in position
    assert np.abs(out_a[ok, :3] - out_b[ok, :3]).max() < 1e-6
    assert np.abs(out_a[ok, 3:] - out_b[ok, 3:]).max() < 1e-9
    rel = np.abs(steps_a - steps_b) / np.maximum(steps_b, 1)
    assert np.median(rel) <= 0.05 and rel.max() <= 0.2
    assert (evals_a[ok] > 0).all() and (evals_b[ok] > 0).all()


def test_noalloc_matches_host_buffer_entry_point_two_calls():
    order = 70
    text = workloads.synthetic_field(order)
    ctx = make_ctx(text, order)

    # call 1: 700 rows, one rectification segment, per-row ballistics
    s1 = workloads.leo_states(700, seed=41)
    b1 = workloads.leo_ballistics(700, seed=41)
    got1 = ctx.propagate_final_noalloc(s1, EPOCH, 5400.0, ballistic=b1)
    ref1 = ctx.propagate_final(s1, EPOCH, 5400.0, ballistic=b1)
    assert (ref1[1] == 0).all()
    check_same(got1, ref1)

    # call 2 right after: fewer rows, other end times, context ballistics, and
    # one invalid row whose status must come from this call
    s2 = workloads.leo_states(300, seed=42)
    s2[17] = [7000.0, 0.0, 0.0, 0.0, 12.0, 0.0]  # hyperbolic: INVALID_INPUT
    tf2 = np.linspace(600.0, 7200.0, 300)
    got2 = ctx.propagate_final_noalloc(s2, EPOCH, tf2)
    ref2 = ctx.propagate_final(s2, EPOCH, tf2)
    assert ref2[1][17] == 3 and (np.delete(ref2[1], 17) == 0).all()
    check_same(got2, ref2)
    assert np.isnan(got2[0][17]).all()


def test_noalloc_rejects_more_rows_than_its_array_holds():
    text = workloads.synthetic_field(8)
    ctx = make_ctx(text, 8)
    n = N.NOALLOC_MAX_TRAJ + 1
    states = np.tile(workloads.leo_states(1, seed=1), (n, 1))
    with pytest.raises(N.NativeError) as e:
        ctx.propagate_final_noalloc(states, EPOCH, 600.0)
    assert e.value.code == N.E_ARG and "no-allocation limit" in str(e.value)
    # the limit itself is accepted
    out, st, _, _ = ctx.propagate_final_noalloc(states[:N.NOALLOC_MAX_TRAJ], EPOCH, 60.0)
    assert (st == 0).all() and np.isfinite(out).all()


def test_noalloc_refuses_forms_it_would_not_run():
    # split precision and the surrogate live in the stage-synchronous engine;
    # the allocation-free path must refuse them, not run plain FP64 instead
    order = 20
    text = workloads.synthetic_field(order)
    cfg = N.default_config()
    cfg.order = order
    cfg.split_degree = 8
    ctx = N.Context(text, cfg)
    s = workloads.leo_states(4, seed=3)
    with pytest.raises(N.NativeError) as e:
        ctx.propagate_final_noalloc(s, EPOCH, 600.0)
    assert e.value.code == N.E_UNSUPPORTED and "split precision" in str(e.value)
    # SRP's eclipse coordinator keeps per-row state the fixed array has no
    # room for: refused too
    cfg.split_degree = 0
    cfg.force_flags |= N.FORCE_SRP
    ctx.set_config(cfg)
    with pytest.raises(N.NativeError) as e:
        ctx.propagate_final_noalloc(s, EPOCH, 600.0)
    assert e.value.code == N.E_UNSUPPORTED and "SRP" in str(e.value)
    # the IAU frame builds its segment table per call: refused as well
    cfg.force_flags &= ~N.FORCE_SRP
    ctx.set_config(cfg)
    ctx.set_frame("iau2006")
    with pytest.raises(N.NativeError) as e:
        ctx.propagate_final_noalloc(s, EPOCH, 600.0)
    assert e.value.code == N.E_UNSUPPORTED and "IAU" in str(e.value)
    # the same context in plain FP64 without SRP, in the GMST frame, runs
    ctx.set_frame("gmst")
    out, st, _, _ = ctx.propagate_final_noalloc(s, EPOCH, 600.0)
    assert (st == 0).all() and np.isfinite(out).all()


def test_noalloc_bits_do_not_depend_on_call_history():
    # the drag sweep fits are built with the context, so a first no-allocation
    # call on a fresh context, one after a host-buffer call and one after the
    # drivers were reset give the same bits
    order = 20
    text = workloads.synthetic_field(order)
    ctx = make_ctx(text, order)
    s = workloads.leo_states(64, seed=44)
    b = workloads.leo_ballistics(64, seed=44)
    first = ctx.propagate_final_noalloc(s, EPOCH, 3000.0, ballistic=b)
    ctx.propagate_final(s, EPOCH, 3000.0, ballistic=b)
    second = ctx.propagate_final_noalloc(s, EPOCH, 3000.0, ballistic=b)
    ctx.set_jb_drivers(None, None)
    third = ctx.propagate_final_noalloc(s, EPOCH, 3000.0, ballistic=b)
    assert (first[1] == 0).all()
    for other in (second, third):
        assert np.array_equal(first[0], other[0]) and np.array_equal(first[1], other[1])
        assert np.array_equal(first[2], other[2]) and np.array_equal(first[3], other[3])


def test_noalloc_kernel_time_is_profiled():
    text = workloads.synthetic_field(8)
    ctx = make_ctx(text, 8)
    ctx.profile(True)
    ctx.propagate_final_noalloc(workloads.leo_states(32, seed=5), EPOCH, 600.0)
    ms, launches = ctx.profile_read()["persistent"]
    ctx.profile(False)
    assert launches == 1 and ms > 0.0
