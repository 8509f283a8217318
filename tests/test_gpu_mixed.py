"""Uneven batch (mixed LEO / MEO / GEO / HEO orbits, uneven durations, drag
only where the perigee is below 2000 km) against the CPU restatement, on
both engines; durations are scaled down from 1 h .. 30 d to 2 min .. 1 d so
the restatement finishes in seconds."""
import numpy as np
import pytest

from bqp_b200 import _native as N
from bqp_b200 import autotune, workloads
from oracle import oracle as O

pytestmark = pytest.mark.gpu

EPOCH = workloads.EPOCH_JD


@pytest.mark.parametrize("engine", ["pipeline", "persistent"])
def test_mixed_orbits_uneven_durations_match_oracle(engine):
    order, eps = 20, 1e-9
    text = workloads.synthetic_field(order)
    states, dur, low = workloads.mixed_states(40, seed=3)
    dur = dur / 30.0
    bal = workloads.mixed_ballistics(low, seed=3)
    cfg = N.default_config()
    cfg.order = order
    cfg.force_flags = N.FORCE_DRAG | N.FORCE_SUN | N.FORCE_MOON
    cfg.eps = eps
    cfg.engine = N.ENGINES[engine]
    ctx = N.Context(text, cfg)
    got, st, steps, evals = ctx.propagate_final(states, EPOCH, dur, ballistic=bal)
    assert (st == 0).all()
    F = O.Force(text, order, drag=True, sun=True, moon=True, atm_model=cfg.atm_model)
    equ, _ = N.eci_to_equinoctial(states)
    d, rst, rsteps, _ = O.propagate_final_batch(F, O.ctrl("dop853", eps=eps), equ, EPOCH, dur, bal)
    assert (rst == 0).all()
    for i in range(len(states)):
        ref = O.equinoc2eci(equ[i], dur[i])[0] + d[i]
        # each solution within ~10 eps per step of the exact one, so two
        # solutions within twice that (as test_adaptive_final_matches_oracle)
        assert np.linalg.norm(got[i, :3] - ref[:3]) <= 2 * max(steps[i], 1) * eps * 10, i
    # accept/reject sequences are chaotic in the last bits: a few steps apart
    # on short, eccentric rows, a few percent on long ones
    assert np.all(np.abs(steps - rsteps) <= np.maximum(5, 0.1 * rsteps))
    # the rows without drag really skip it, and durations differ by 720x
    assert (bal[~low, 0] == 0).all() and dur.max() / dur.min() > 100


def test_autotuner_picks_a_measured_candidate():
    order = 20
    text = workloads.synthetic_field(order)
    states, dur, low = workloads.mixed_states(2048, seed=5)
    bal = workloads.mixed_ballistics(low, seed=5)
    cfg = N.default_config()
    cfg.order = order
    cfg.force_flags = N.FORCE_DRAG | N.FORCE_SUN | N.FORCE_MOON
    best, results = autotune.tune(text, cfg, states, EPOCH, dur, bal, sample=1024, trial_s=300.0)
    assert results and all(r["ok"] == 1024 for r in results)
    top = max(results, key=lambda r: r["evals_per_s"])
    assert best.engine == N.ENGINES[top["engine"]] and best.gravity_slots == top["gravity_slots"]
    again, cached = autotune.tune(text, cfg, states, EPOCH, dur, bal, sample=1024, trial_s=300.0)
    assert cached is None and again.gravity_threads == best.gravity_threads
