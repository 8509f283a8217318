"""Launch-shape autotuner for a propagation workload.

Times each candidate (engine, gravity threads per CTA, rows per gravity
thread) on a sample of the batch over a short arc and keeps the fastest
by force evaluations per second; the choice is cached per (device, field
order, batch-size bucket) for the life of the process.

    python -m bqp_b200.autotune --workload mixed --n 32768
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import _native as N
from . import workloads as W

CANDIDATES = [
    ("pipeline", 256, 4), ("pipeline", 256, 2), ("pipeline", 128, 4), ("pipeline", 256, 1),
    ("persistent", 256, 4),
]
_cache: dict = {}


def _bucket(n: int) -> int:
    return 1 << max(10, int(np.ceil(np.log2(max(n, 1)))))


def tune(text: str, cfg, states, epoch_jd, tf, ballistic=None, sample: int = 16384, trial_s: float = 1800.0,
         candidates=None, device_key: str = "cuda:0"):
    """Returns (best_cfg, results).  `cfg` is copied; the trial propagates
    min(n, sample) rows for min(tf, trial_s) seconds per candidate."""
    n = len(states)
    key = (device_key, int(cfg.order), int(cfg.split_degree), _bucket(n))
    if key in _cache:
        best = _cache[key]
        out = N.ForceConfig.from_buffer_copy(cfg)
        out.engine, out.gravity_threads, out.gravity_slots = N.ENGINES[best[0]], best[1], best[2]
        return out, None
    idx = np.linspace(0, n - 1, min(n, sample)).astype(np.int64)
    s = np.asarray(states)[idx]
    tfa = np.minimum(np.broadcast_to(tf, (n,))[idx], trial_s)
    bal = None if ballistic is None else np.asarray(ballistic)[idx]
    results = []
    for engine, threads, slots in candidates or CANDIDATES:
        c = N.ForceConfig.from_buffer_copy(cfg)
        c.engine, c.gravity_threads, c.gravity_slots = N.ENGINES[engine], threads, slots
        if engine == "persistent" and (c.split_degree or c.drag_fp32):
            continue
        ctx = N.Context(text, c)
        ctx.propagate_final(s[:256], epoch_jd, np.minimum(tfa[:256], 60.0), ballistic=None if bal is None else bal[:256])
        t0 = time.perf_counter()
        _, st, _, ev = ctx.propagate_final(s, epoch_jd, tfa, ballistic=bal)
        dt = time.perf_counter() - t0
        ctx.close()
        results.append({"engine": engine, "gravity_threads": threads, "gravity_slots": slots,
                        "evals_per_s": float(ev.sum() / dt), "ok": int((st == 0).sum())})
    best = max(results, key=lambda r: r["evals_per_s"])
    _cache[key] = (best["engine"], best["gravity_threads"], best["gravity_slots"])
    out = N.ForceConfig.from_buffer_copy(cfg)
    out.engine, out.gravity_threads, out.gravity_slots = (N.ENGINES[best["engine"]], best["gravity_threads"],
                                                          best["gravity_slots"])
    return out, results


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="mixed", choices=["mixed", "leo"])
    ap.add_argument("--n", type=int, default=32768)
    ap.add_argument("--order", type=int, default=70)
    ap.add_argument("--sample", type=int, default=16384)
    ap.add_argument("--trial-s", type=float, default=1800.0)
    ap.add_argument("--run", action="store_true", help="then propagate the whole batch with the choice")
    ap.add_argument("--eps", type=float, default=1e-12, help="absolute tolerance, km (DOP853)")
    ap.add_argument("--atm-model", type=int, default=4, choices=[4, 5, 6, 7], help="JB2008 profile")
    args = ap.parse_args()
    from .accuracy import config
    text = W.synthetic_field(args.order)
    if args.workload == "mixed":
        states, dur, low = W.mixed_states(args.n, seed=0)
        bal = W.mixed_ballistics(low, seed=0)
    else:
        states = W.leo_states(args.n, seed=0)
        dur = np.full(args.n, 5400.0)
        bal = W.leo_ballistics(args.n, seed=0)
    cfg = config(args.order, args.eps)
    cfg.atm_model = args.atm_model
    best, results = tune(text, cfg, states, W.EPOCH_JD, dur, bal, args.sample, args.trial_s)
    out = {"workload": args.workload, "n": args.n, "eps_km": args.eps, "atm_model": args.atm_model,
           "trials": results,
           "choice": {"engine": [k for k, v in N.ENGINES.items() if v == best.engine][0],
                      "gravity_threads": best.gravity_threads, "gravity_slots": best.gravity_slots}}
    if args.run:
        ctx = N.Context(text, best)
        t0 = time.perf_counter()
        _, st, _, ev = ctx.propagate_final(states, W.EPOCH_JD, dur, ballistic=bal)
        dt = time.perf_counter() - t0
        out["run"] = {"wall_s": dt, "evals": int(ev.sum()), "evals_per_s": float(ev.sum() / dt),
                      "trajectory_days_per_s": float(dur.sum() / 86400.0 / dt), "ok": int((st == 0).sum()),
                      "status_counts": {int(k): int(v) for k, v in zip(*np.unique(st, return_counts=True))}}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
