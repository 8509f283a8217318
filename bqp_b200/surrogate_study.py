"""The learned gravity surrogate at the C5 scale: train it on the GPU on
samples of an exact field, then measure its field error and its evaluation
rate against the exact kernel, on the GPU.

    python -m bqp_b200.surrogate_study --order 120 --samples 16777216 --epochs 4

Reported: training time and loss per epoch; on held-out positions (radius
U[6578, 7578] km, uniform on the sphere) the RMS and max error of the
degree > 8 residual with the network and without it (the low-degree field
alone), relative to the RMS residual, and the error relative to the full
field; evaluation rates (force evaluations/s, device-resident positions, CUDA
events) of the exact FP64 kernel and of the low-degree field + network, and
the network's tensor-core GEMM rate.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import _native as N
from . import workloads as W


def _ctx(text, order):
    cfg = N.default_config()
    cfg.order = order
    return N.Context(text, cfg)


def _timed(torch, fn, reps=5):
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def propagation(text, order, sur_ctx, n, seconds, eps_ref=1e-12, eps_form=1e-9, limit_s=120.0, check=1e-3):
    """n LEO rows (the bench distributions) over `seconds` with DOP853,
    gravity + Sun/Moon.  Reference: the exact FP64 field at eps_ref.  Forms at
    eps_form: the exact field, the degree-8 field alone, the surrogate (its
    BF16-level field error drives the step controller at a 1e-12 km
    tolerance, so it runs at its own) and the surrogate with the per-step
    residual check at `check`.  Wall-clock rates and final-position
    differences from the reference (m); every run is limited to limit_s."""
    states = W.leo_states(n, seed=5)
    out = {"rows": n, "seconds": seconds, "eps_ref": eps_ref, "eps_form": eps_form, "check": check}
    res = {}
    for name, order_, sur, eps, chk in (("exact_ref", order, False, eps_ref, 0.0),
                                        ("exact", order, False, eps_form, 0.0),
                                        ("degree8", N.SURROGATE_DEGREE, False, eps_form, 0.0),
                                        ("surrogate", order, True, eps_form, 0.0),
                                        ("surrogate_checked", order, True, eps_form, check)):
        c = sur_ctx if sur else _ctx(text, order_)
        cfg = N.default_config()
        cfg.order = order_
        cfg.force_flags = N.FORCE_SUN | N.FORCE_MOON
        cfg.eps = eps
        cfg.surrogate = int(sur)
        cfg.surrogate_check = chk
        cfg.max_kernel_seconds = limit_s
        c.set_config(cfg)
        c.propagate_final(states[:1024], W.EPOCH_JD, 60.0)  # warm-up
        t0 = time.perf_counter()
        r, st, _, ev = c.propagate_final(states, W.EPOCH_JD, seconds)
        wall = time.perf_counter() - t0
        res[name] = r
        out[name] = {"wall_s": wall, "evals": int(ev.sum()), "evals_per_s": float(ev.sum() / wall),
                     "trajectory_days_per_s": n * seconds / 86400.0 / wall, "ok": int((st == 0).sum())}
    for name in ("exact", "degree8", "surrogate", "surrogate_checked"):
        d = np.linalg.norm(res[name][:, :3] - res["exact_ref"][:, :3], axis=1) * 1e3
        out[name]["err_m_rms"] = float(np.sqrt(np.mean(d ** 2)))
        out[name]["err_m_max"] = float(d.max())
    return out


def study(order=120, samples=1 << 24, epochs=4, batch=16384, lr=2e-3, n_eval=200000, n_rate=1 << 20, seed=1,
          n_prop=0, prop_s=5400.0, eps_form=1e-9, check=1e-3):
    import torch
    text = W.synthetic_field(order)
    ctx = _ctx(text, order)
    stream = torch.cuda.current_stream().cuda_stream
    ctx.set_stream(stream)
    t0 = time.perf_counter()
    loss = ctx.surrogate_train(samples=samples, epochs=epochs, batch=batch, lr=lr, seed=seed)
    train_s = time.perf_counter() - t0

    rng = np.random.default_rng(seed + 100)
    r = rng.uniform(6578.0, 7578.0, n_eval)
    u = rng.normal(size=(n_eval, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    pos = u * r[:, None]
    full = ctx.gravity(pos)[0]
    low = _ctx(text, N.SURROGATE_DEGREE).gravity(pos)[0]
    surr = ctx.surrogate_infer(pos, add_low=True)
    res = full - low
    rms_res = float(np.sqrt(np.mean(np.sum(res ** 2, axis=1))))
    e_with = np.linalg.norm(full - surr, axis=1)
    e_without = np.linalg.norm(res, axis=1)
    gnorm = np.linalg.norm(full, axis=1)

    # rates on device-resident positions
    dev = torch.device("cuda")
    rr = rng.uniform(6578.0, 7578.0, n_rate)
    uu = rng.normal(size=(n_rate, 3))
    uu /= np.linalg.norm(uu, axis=1, keepdims=True)
    d_pos = torch.tensor(uu * rr[:, None], device=dev)
    d_acc = torch.empty_like(d_pos)
    ms_exact = _timed(torch, lambda: ctx.gravity_device(n_rate, d_pos.data_ptr(), d_acc.data_ptr()))
    ms_surr = _timed(torch, lambda: ctx.surrogate_infer_device(n_rate, d_pos.data_ptr(), d_acc.data_ptr(), True))
    gemm_flops = 3 * 2 * 256 * 256 * n_rate
    prop = propagation(text, order, ctx, n_prop, prop_s, eps_form=eps_form, check=check) if n_prop else None
    return {
        "propagation": prop,
        "order": order, "samples": samples, "epochs": epochs, "batch": batch, "train_s": train_s,
        "loss_per_epoch": [float(v) for v in loss],
        "eval_points": n_eval,
        "residual_rms_km_s2": rms_res,
        "with_network": {"rms_rel_to_residual": float(np.sqrt(np.mean(e_with ** 2))) / rms_res,
                         "max_rel_to_residual_rms": float(e_with.max()) / rms_res,
                         "max_rel_to_field": float((e_with / gnorm).max())},
        "without_network": {"rms_rel_to_residual": float(np.sqrt(np.mean(e_without ** 2))) / rms_res,
                            "max_rel_to_field": float((e_without / gnorm).max())},
        "rate_points": n_rate,
        "exact_fp64_evals_per_s": n_rate / (ms_exact * 1e-3),
        "surrogate_evals_per_s": n_rate / (ms_surr * 1e-3),
        "surrogate_gemm_tflops": gemm_flops / (ms_surr * 1e-3) / 1e12,
    }


def infer_probe(n: int, order: int = 20, samples: int = 1 << 20) -> dict:
    """The capture case of the fused inference kernel: a surrogate trained for
    one epoch on a 20x20 field, then three device-resident inference calls
    on n positions (the launches a profiler captures)."""
    import torch

    text = W.synthetic_field(order)
    ctx = _ctx(text, order)
    ctx.surrogate_train(samples=samples, epochs=1, batch=8192)
    rng = np.random.default_rng(3)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    pos = d * rng.uniform(6578.0, 7578.0, n)[:, None]
    d_pos = torch.tensor(pos, device="cuda", dtype=torch.float64)
    d_acc = torch.empty_like(d_pos)
    for _ in range(3):
        ctx.surrogate_infer_device(n, d_pos.data_ptr(), d_acc.data_ptr())
    torch.cuda.synchronize()
    return {"positions": n, "calls": 3, "finite": bool(torch.isfinite(d_acc).all().item())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--infer-probe", type=int, default=0,
                    help="only the inference capture case: one-epoch 20x20 surrogate, 3 calls on this many positions")
    ap.add_argument("--order", type=int, default=120)
    ap.add_argument("--samples", type=int, default=1 << 24)
    ap.add_argument("--epochs", type=int, default=4)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--propagate", type=int, default=0, help="rows of the propagation comparison (0: none)")
    ap.add_argument("--prop-seconds", type=float, default=5400.0)
    ap.add_argument("--eps-form", type=float, default=1e-9)
    ap.add_argument("--check", type=float, default=1e-3, help="surrogate_check of the checked propagation form")
    args = ap.parse_args()
    if args.infer_probe:
        print(json.dumps(infer_probe(args.infer_probe)), flush=True)
        return
    print(json.dumps(study(args.order, args.samples, args.epochs, args.batch, args.lr, n_prop=args.propagate,
                           prop_s=args.prop_seconds, eps_form=args.eps_form, check=args.check)), flush=True)


if __name__ == "__main__":
    main()
