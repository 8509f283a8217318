"""Position error of a propagation form against the FP64 form at a tight
tolerance, over a long arc (default 7 days), on the GPU.

The split-precision forms (harmonic degrees above d in FP32, optionally the
JB2008 density in FP32) add rounding noise of ~1e-14 km/s^2 to the force; at
the plain form's 1e-12 km tolerance that noise drives the step controller, so
each form is run at its own tolerance and judged by where its trajectories
end up.  The reference is the stage-synchronous FP64 form at eps = 1e-12 km,
itself checked against the CPU restatement by the test suite.

    python -m bqp_b200.accuracy --n 512 --days 7 --split-degree 8 --eps 1e-10
    python -m bqp_b200.accuracy --n 512 --days 7 --methods vern7 vern9 --eps 1e-10 1e-9

With ``--methods`` the forms are the plain FP64 form with each named stepper
at each tolerance (the reference stays DOP853 at 1e-12 km).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import _native as N
from . import workloads as W

DRIVERS = (150.0,) * 8 + (20.0,)


def config(order=70, eps=1e-12, split_degree=0, drag_fp32=False, drag=True, method="dop853"):
    cfg = N.default_config()
    cfg.order = order
    cfg.force_flags = (N.FORCE_DRAG if drag else 0) | N.FORCE_SUN | N.FORCE_MOON
    cfg.atm_model = 4
    cfg.method = N.METHODS[method]
    cfg.error_control = 0
    cfg.eps = eps
    cfg.dt_max = 300.0
    for i, v in enumerate(DRIVERS):
        cfg.jb_drivers[i] = v
    cfg.max_kernel_seconds = 3000.0
    cfg.split_degree = split_degree
    cfg.drag_fp32 = int(drag_fp32)
    return cfg


def run_form(text, states, bal, tf, cfg):
    ctx = N.Context(text, cfg)
    t0 = time.perf_counter()
    out, st, steps, evals = ctx.propagate_final(states, W.EPOCH_JD, tf, ballistic=bal)
    wall = time.perf_counter() - t0
    ctx.close()
    return out, st, steps, evals, wall


def compare(n=512, days=7.0, order=70, seed=0, forms=None, ref_eps=1e-12):
    """Final-position error (m) of each form against FP64 at ref_eps.

    forms: list of dicts with keys eps, split_degree, drag_fp32 (and a name).
    Rows are the bench workload's distributions (altitude U[400, 1200] km).
    """
    text = W.synthetic_field(order)
    states = W.leo_states(n, seed=seed)
    bal = W.leo_ballistics(n, seed=seed)
    tf = days * 86400.0
    ref, rst, rsteps, revals, rwall = run_form(text, states, bal, tf, config(order, ref_eps))
    alt = np.linalg.norm(states[:, :3], axis=1) - 6378.137
    rows = []
    for f in forms or []:
        out, st, steps, evals, wall = run_form(text, states, bal, tf,
                                               config(order, f["eps"], f.get("split_degree", 0),
                                                      f.get("drag_fp32", False), method=f.get("method", "dop853")))
        ok = (st == 0) & (rst == 0)
        err_m = np.linalg.norm(out[ok, :3] - ref[ok, :3], axis=1) * 1e3
        low = ok & (alt < 500.0)
        rows.append({
            "form": f.get("name", ""), "method": f.get("method", "dop853"), "eps": f["eps"],
            "split_degree": f.get("split_degree", 0),
            "drag_fp32": bool(f.get("drag_fp32", False)), "ok": int(ok.sum()), "n": n,
            "err_m_max": float(err_m.max()) if err_m.size else None,
            "err_m_median": float(np.median(err_m)) if err_m.size else None,
            "err_m_p99": float(np.percentile(err_m, 99)) if err_m.size else None,
            "err_m_max_below_500km": float((np.linalg.norm(out[low, :3] - ref[low, :3], axis=1) * 1e3).max())
            if low.any() else None,
            "evals": int(evals.sum()), "evals_ratio_to_ref": float(evals.sum() / revals.sum()),
            "wall_s": wall,
        })
    return {"n": n, "days": days, "order": order, "ref": {"eps": ref_eps, "evals": int(revals.sum()),
                                                         "ok": int((rst == 0).sum()), "wall_s": rwall},
            "forms": rows}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--days", type=float, default=7.0)
    ap.add_argument("--order", type=int, default=70)
    ap.add_argument("--split-degree", type=int, default=8)
    ap.add_argument("--drag-fp32", action="store_true")
    ap.add_argument("--eps", type=float, nargs="+", default=[1e-12, 1e-11, 1e-10, 1e-9])
    ap.add_argument("--fp64-too", action="store_true", help="also the FP64 form at each eps")
    ap.add_argument("--methods", nargs="+", choices=sorted(N.METHODS),
                    help="plain FP64 forms with these steppers instead of the split forms")
    args = ap.parse_args()
    forms = []
    for e in args.eps:
        if args.methods:
            forms += [{"name": f"plain FP64 {m}", "eps": e, "method": m} for m in args.methods]
            continue
        forms.append({"name": f"split d>{args.split_degree}", "eps": e, "split_degree": args.split_degree,
                      "drag_fp32": args.drag_fp32})
        if args.fp64_too:
            forms.append({"name": "plain FP64", "eps": e})
    print(json.dumps(compare(args.n, args.days, args.order, forms=forms)), flush=True)


if __name__ == "__main__":
    main()
