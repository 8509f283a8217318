"""Benchmark of the batched orbit propagator (one JSON line on rank 0).

Workload (the 70x70 + drag configuration): 65,536 LEO states (altitude U[400,
1200] km, e U[0, 0.02], i U[0, 98] deg, angles U[0, 360) deg, seed 0), a
synthetic 70x70 normalised Kaula-rule field, JB2008 drag (F10.7 = S10 = M10 =
Y10 = 150, dTc = 20 K), A/m U[0.005, 0.05] m^2/kg, Cd 2.2, Sun/Moon point
masses, DOP853 with absolute tolerance 1e-12 (the reference's smallest
eps, integrator.rs:427), dt_max 300 s.

One step = one Encke rectification segment (5400 s) of the whole batch: the
7-day arc is 112 such segments, and each call continues from the previous
call's output exactly as the reference's segment loop does
(integrator.rs:3418-3560).  Metric: force (RHS) evaluations per second, counted
by the device per trajectory.

  value  device-resident inputs, each step timed with CUDA events
  e2e    the same steps through the host-buffer C ABI call
         (bqp_propagate_final): H2D of the inputs and D2H of the results
         inside the timed region
  roofline  the gravity kernel (pl_gravity), FP64: algorithmic flops =
         force evals x F(70) (the reference gravity algorithm's flop count,
         F(N) = 9(N+2)(N+3)/2 + 13N(N+1) + 9(N+1) + 60, FMA = 2) over the
         kernel's summed CUDA-event time in the timed steps; peak = cuBLAS
         DGEMM measured in this run
  cpu_baseline  the C++ oracle (restatement of the reference CPU path) on a
         bounded sample, all host cores

  forms  (N = 1 only) the propagation forms the metric compares with plain
         FP64: split precision at eps 1e-11 (degrees above 8, 16, 32 in FP32),
         plain FP64 at eps 1e-10 and Vern9 at eps 1e-10 -- each form's force
         evaluations/s and trajectory-days/s on the full batch, and its 7-day
         final-position error against plain FP64 at eps 1e-12 on 512 rows
         (``--no-forms`` skips it)

``--impl reference`` times that CPU implementation alone (rank 0) on the same
workload and prints its line.  ``--atm-model 7`` measures the reference's
default (fitted) JB2008 profile instead of the exact model; ``--srp`` adds
solar radiation pressure through the binary-eclipse coordinator (cr 1.3) on
both arms; ``--frame iau2006`` takes the Earth-fixed frame from the IAU
2006/2000A segments (zero EOP; the reference's production frame) instead of
the GMST rotation, on both arms (the oracle evaluates the same segments).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "force evals/s @70x70+drag: plain FP64 vs split/surrogate at ≤1 m 7-day err"
UNIT = "force_evals/s"
ORDER = 70
N_TRAJ = 65536
SEGMENT_S = 5400.0
EPS = 1e-12
DRIVERS = (150.0,) * 8 + (20.0,)


def form_name(args) -> str:
    if not args.split_degree and not args.drag_fp32:
        return "plain FP64"
    parts = []
    if args.split_degree:
        parts.append(f"harmonic degrees > {args.split_degree} in FP32")
    if args.drag_fp32:
        parts.append("JB2008 density in FP32")
    return "split: " + ", ".join(parts)


def f_of_n(n: int) -> float:
    return 9 * (n + 2) * (n + 3) / 2 + 13 * n * (n + 1) + 9 * (n + 1) + 60


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_TRAJ)
    ap.add_argument("--cpu-sample", type=int, default=256, help="trajectories in the CPU baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--segment", type=float, default=SEGMENT_S,
                    help="seconds propagated per step (5400 = one Encke segment; smaller for profiling)")
    ap.add_argument("--engine", default="pipeline", choices=["pipeline", "persistent"])
    ap.add_argument("--gravity-threads", type=int, default=256)
    ap.add_argument("--split-degree", type=int, default=0,
                    help="split precision: harmonic degrees above this in FP32 (0: plain FP64)")
    ap.add_argument("--drag-fp32", action="store_true", help="split precision: JB2008 density in FP32")
    ap.add_argument("--method", default="dop853", choices=["dop853", "vern7", "vern9", "dopri5"],
                    help="stepper (the metric's workload: dop853 at eps 1e-12)")
    ap.add_argument("--eps", type=float, default=EPS, help="absolute tolerance, km")
    ap.add_argument("--atm-model", type=int, default=4, choices=[4, 5, 6, 7],
                    help="JB2008 profile (4 exact: the metric's workload; 7 the reference's Python default)")
    ap.add_argument("--srp", action="store_true",
                    help="solar radiation pressure with binary eclipse (cr 1.3) on every row, both arms")
    ap.add_argument("--frame", default="gmst", choices=["gmst", "iau2006"],
                    help="Earth-fixed frame: GMST z-rotation, or the IAU 2006/2000A segments (zero EOP)")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the forms block (split precision and other steppers against plain FP64)")
    ap.add_argument("--forms-rows", type=int, default=512, help="rows of the 7-day accuracy runs of the forms")
    ap.add_argument("--forms-days", type=float, default=7.0)
    return ap.parse_args(argv)


# ------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# -------------------------------------------------------------- workload
def make_workload(n: int, seed: int = 0):
    from bqp_b200 import workloads as W

    states = W.leo_states(n, seed=seed)
    bal = W.leo_ballistics(n, seed=seed)
    return W.synthetic_field(ORDER), states, bal, W.EPOCH_JD


def make_config(engine="pipeline", gravity_threads=256, split_degree=0, drag_fp32=False, method="dop853",
                eps=EPS, atm_model=4, srp=False):
    from bqp_b200 import _native as N

    cfg = N.default_config()
    cfg.split_degree = split_degree
    cfg.drag_fp32 = int(drag_fp32)
    cfg.engine = N.ENGINES[engine]
    cfg.gravity_threads = gravity_threads
    cfg.order = ORDER
    cfg.force_flags = N.FORCE_DRAG | N.FORCE_SUN | N.FORCE_MOON | (N.FORCE_SRP if srp else 0)
    cfg.cr = 1.3
    cfg.atm_model = atm_model
    cfg.method = N.METHODS[method]
    cfg.error_control = 0
    cfg.eps = eps
    cfg.dt_max = 300.0
    for i, v in enumerate(DRIVERS):
        cfg.jb_drivers[i] = v
    cfg.max_kernel_seconds = 300.0
    return cfg


def bench_config(args) -> dict:
    """The workload's description, the same dict on both arms (the reference
    arm's bounded sample is reported beside it, in its own key)."""
    srp = " + SRP with binary eclipse" if args.srp else ""
    srp += ", IAU 2006/2000A Earth-fixed frame" if args.frame == "iau2006" else ""
    return {"workload": f"{args.n} LEO states per GPU, 70x70 Kaula field + JB2008 drag + Sun/Moon{srp}, "
                        f"{args.method.upper()} eps {args.eps:g}, {args.segment:g} s of the arc per step",
            "form": form_name(args), "order": ORDER, "trajectories_per_gpu": args.n, "segment_s": args.segment,
            "method": args.method, "eps_km": args.eps, "atm_model": args.atm_model, "srp": bool(args.srp),
            "frame": args.frame,
            "l2": "256 MiB write between timed steps"}


def cpu_reference(sample: int, threads: int, segments: int = 1, method: str = "dop853", eps: float = EPS,
                  segment_s: float = SEGMENT_S, atm_model: int = 4, srp: bool = False, frame: str = "gmst"):
    """Time the CPU oracle (restatement of the reference path) on the first
    `sample` trajectories of the workload for `segments` segments, all
    threads.  Only the oracle runs here: the elements come from its own
    ECI -> equinoctial conversion, so this path loads no product library."""
    from oracle import oracle as O

    text, states, bal, epoch = make_workload(N_TRAJ)
    states, bal = np.ascontiguousarray(states[:sample]), np.ascontiguousarray(bal[:sample])
    equ = np.array([O.eci2equinoc(s)[0] for s in states])
    F = O.Force(text, ORDER, drag=True, sun=True, moon=True, drivers=DRIVERS, atm_model=atm_model)
    ctl = O.ctrl(method, eps=eps, dt_max=300.0)
    if srp:
        F.set_srp(True, 1.3)
    if frame == "iau2006":
        # the frame segments are an input of the force model: built by the
        # library's host authority (zero EOP), outside the timed region
        from bqp_b200 import _native as N

        auth = N.FrameAuthority()
        tai0 = N.tai_seconds(epoch)[0]
        keys, segs = auth.segments(tai0 - 1800.0, tai0 + segment_s * segments + 1800.0)
        F.set_frame(keys, segs, auth.intervals()["raw"])
    t0 = time.perf_counter()
    if srp:
        _, _, st, steps, evals, _ = O.propagate_srp_batch(F, ctl, equ, epoch, segment_s * segments, bal,
                                                          threads=threads)
    else:
        _, st, steps, evals = O.propagate_final_batch(F, ctl, equ, epoch, segment_s * segments, bal, threads=threads)
    dt = time.perf_counter() - t0
    return float(evals.sum()) / dt, dt, int(evals.sum()), int((st == 0).sum())


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    evals_s = []
    for i in range(args.warmup + args.steps):
        v, dt, ev, ok = cpu_reference(args.cpu_sample, threads, method=args.method, eps=args.eps,
                                      segment_s=args.segment, atm_model=args.atm_model, srp=args.srp,
                                      frame=args.frame)
        if i >= args.warmup:
            evals_s.append((v, dt))
    value = statistics.median(v for v, _ in evals_s)
    ms = statistics.median(dt for _, dt in evals_s) * 1e3
    sample = f"{args.cpu_sample} of the {args.n} trajectories, one {args.segment:g} s segment per step"
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": bench_config(args),
        "sample": {"trajectories": args.cpu_sample, "of": args.n, "segments_per_step": 1},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ ours
# DRAM bytes (read + write) per launch of the dominant kernel from one ncu
# capture (profiles/pl_gravity_70x70.md: 37,888 rows, one launch), scaled by
# the rows one launch of this run processes.
TRAFFIC_CAPTURE = {"gravity": (1895424.0, 37888)}


def traffic_per_launch(kernel: str, rows: int):
    if kernel not in TRAFFIC_CAPTURE:
        return None
    b, r = TRAFFIC_CAPTURE[kernel]
    return b * rows / r


def fp64_peak_tflops(torch, dev):
    """Measured FP64 peak: cuBLAS DGEMM 8192^3, best of 5 (CUDA events)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    b = torch.randn(8192, 8192, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def combine_ranks(t_local, evals_local, world, device):
    """Whole-job figures of a weak-scaled run: the slowest rank's time and the
    evaluations of all ranks (every rank takes both collectives, in this
    order).  One rank: the local figures."""
    if world <= 1:
        return float(t_local), float(evals_local)
    import torch
    import torch.distributed as dist

    tt = torch.tensor([float(t_local)], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    ev = torch.tensor([float(evals_local)], device=device, dtype=torch.float64)
    dist.all_reduce(ev, op=dist.ReduceOp.SUM)
    return float(tt.item()), float(ev.item())


# ------------------------------------------------------------------ forms
# The propagation forms the metric compares with plain FP64 (DOP853, eps
# 1e-12 km): split precision (spherical-harmonic degrees above d in FP32) at
# the tolerance its FP32 noise allows, and the higher-order Verner stepper.
FORMS = [
    {"name": "plain FP64, DOP853 eps 1e-10", "method": "dop853", "eps": 1e-10, "split_degree": 0},
    {"name": "split d>8, DOP853 eps 1e-11", "method": "dop853", "eps": 1e-11, "split_degree": 8},
    {"name": "split d>16, DOP853 eps 1e-11", "method": "dop853", "eps": 1e-11, "split_degree": 16},
    {"name": "split d>32, DOP853 eps 1e-11", "method": "dop853", "eps": 1e-11, "split_degree": 32},
    {"name": "plain FP64, Vern9 eps 1e-10", "method": "vern9", "eps": 1e-10, "split_degree": 0},
]


def form_throughput(f, text, states, bal, epoch, seg, dev, warmup=1, steps=2):
    """Force evaluations/s and trajectory-days/s of one form on the full
    batch, device-resident, `steps` segments timed with CUDA events."""
    import torch

    from bqp_b200 import _native as N

    n = states.shape[0]
    ctx = N.Context(text, make_config(split_degree=f["split_degree"], method=f["method"], eps=f["eps"]))
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    with torch.cuda.stream(stream):
        a = torch.tensor(states, device=dev, dtype=torch.float64)
        b = torch.empty_like(a)
        d_bal = torch.tensor(bal, device=dev, dtype=torch.float64)
        d_tf = torch.full((n,), seg, device=dev, dtype=torch.float64)
        d_st = torch.empty(n, device=dev, dtype=torch.int32)
        d_steps = torch.empty(n, device=dev, dtype=torch.int64)
        d_ev = torch.empty(n, device=dev, dtype=torch.int64)
        eps_k = [torch.full((n,), epoch + k * seg / 86400.0, device=dev, dtype=torch.float64)
                 for k in range(warmup + steps)]
        flush = torch.empty(256 * 1024 * 1024 // 4, device=dev, dtype=torch.float32)
        total = torch.zeros((), device=dev, dtype=torch.int64)
    stream.synchronize()
    ms = 0.0
    for k in range(warmup + steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.propagate_final_device(a.data_ptr(), eps_k[k].data_ptr(), d_tf.data_ptr(), b.data_ptr(),
                                   d_st.data_ptr(), d_steps.data_ptr(), d_ev.data_ptr(), n=n,
                                   d_ballistic=d_bal.data_ptr())
        e1.record(stream)
        if k >= warmup:
            with torch.cuda.stream(stream):
                total += d_ev.sum()
        stream.synchronize()
        if k >= warmup:
            ms += e0.elapsed_time(e1)
        a, b = b, a
    ok = float((d_st == 0).float().mean().item())
    ev = int(total.item())
    ctx.close()
    return {"force_evals_per_s": ev / (ms * 1e-3), "trajectory_days_per_s": n * seg * steps / 86400.0 / (ms * 1e-3),
            "evals_per_step": ev / steps, "status_ok_fraction": ok}


def form_accuracy_runs(forms, text, states, bal, epoch, days):
    """Final states of every form (and of plain FP64 at eps 1e-12, the
    reference) after `days`, each on its own context and stream, all at
    once: these small batches are latency-bound, so they share the GPU."""
    import threading

    import torch

    from bqp_b200 import _native as N

    results = {}

    def run(key, f):
        cfg = make_config(split_degree=f["split_degree"], method=f["method"], eps=f["eps"])
        cfg.max_kernel_seconds = 3000.0
        ctx = N.Context(text, cfg)
        stream = torch.cuda.Stream()
        ctx.set_stream(stream.cuda_stream)
        t0 = time.perf_counter()
        out, st, steps, ev = ctx.propagate_final(states, epoch, days * 86400.0, ballistic=bal)
        results[key] = (out, st, ev, time.perf_counter() - t0)
        ctx.close()

    jobs = [("ref", {"method": "dop853", "eps": EPS, "split_degree": 0})] + list(enumerate(forms))
    threads = [threading.Thread(target=run, args=job) for job in jobs]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    return results


def run_forms(args, text, states, bal, epoch, dev, plain):
    rows = np.linspace(0, states.shape[0] - 1, args.forms_rows).astype(np.int64)
    sub_s, sub_b = np.ascontiguousarray(states[rows]), np.ascontiguousarray(bal[rows])
    t0 = time.perf_counter()
    acc = form_accuracy_runs(FORMS, text, sub_s, sub_b, epoch, args.forms_days)
    acc_wall = time.perf_counter() - t0
    ref_out, ref_st, ref_ev, ref_wall = acc["ref"]
    out = []
    for i, f in enumerate(FORMS):
        thr = form_throughput(f, text, states, bal, epoch, args.segment, dev)
        fo, fst, fev, fwall = acc[i]
        ok = (fst == 0) & (ref_st == 0)
        err_m = np.linalg.norm(fo[ok, :3] - ref_out[ok, :3], axis=1) * 1e3
        emax = float(err_m.max()) if err_m.size else None
        out.append({
            "form": f["name"], "method": f["method"], "eps_km": f["eps"], "split_degree": f["split_degree"],
            **{k: v for k, v in thr.items()},
            "vs_plain_force_evals_per_s": thr["force_evals_per_s"] / plain["force_evals_per_s"],
            "vs_plain_trajectory_days_per_s": thr["trajectory_days_per_s"] / plain["trajectory_days_per_s"],
            "err_m_max": emax, "err_m_median": float(np.median(err_m)) if err_m.size else None,
            "within_1m": bool(emax is not None and emax <= 1.0 and ok.all()),
            "evals_vs_plain_7d": float(fev.sum() / ref_ev.sum()), "rows_ok": int(ok.sum()),
        })
    return {"reference": f"plain FP64, DOP853 eps {EPS:g} km on the same rows",
            "accuracy_rows": int(rows.size), "accuracy_days": args.forms_days,
            "accuracy_wall_s": acc_wall, "reference_evals_7d": int(ref_ev.sum()),
            "throughput": f"{states.shape[0]} rows, one {args.segment:g} s segment per step, 2 timed steps "
                          "after 1 warm-up, device-resident",
            "forms": out}


def run_ours(args):
    import torch
    import torch.distributed as dist

    from bqp_b200 import _native as N

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)

    text, states, bal, epoch = make_workload(args.n, seed=rank)
    cfg = make_config(args.engine, args.gravity_threads, args.split_degree, args.drag_fp32, args.method, args.eps,
                      args.atm_model, args.srp)
    ctx = N.Context(text, cfg)
    seg = args.segment
    if args.frame == "iau2006":
        # segments for every step's span, built once: the device calls stay
        # asynchronous (no per-call epoch readback)
        ctx.set_frame("iau2006")
        ctx.set_frame_span(epoch - 1.0, epoch + (args.warmup + 2 * args.steps + 2) * seg / 86400.0 + 1.0)
    stream = torch.cuda.Stream(device=dev)
    ctx.set_stream(stream.cuda_stream)
    n = args.n

    # device-resident state: chain segments in place (out of step k = in of k+1)
    with torch.cuda.stream(stream):
        d_a = torch.tensor(states, device=dev, dtype=torch.float64)
        d_b = torch.empty_like(d_a)
        d_bal = torch.tensor(bal, device=dev, dtype=torch.float64)
        d_tf = torch.full((n,), seg, device=dev, dtype=torch.float64)
        d_status = torch.empty(n, device=dev, dtype=torch.int32)
        d_steps = torch.empty(n, device=dev, dtype=torch.int64)
        d_evals = torch.empty(n, device=dev, dtype=torch.int64)
        flush = torch.empty(256 * 1024 * 1024 // 4, device=dev, dtype=torch.float32)
    epochs = [epoch + k * seg / 86400.0 for k in range(args.warmup + 2 * args.steps + 1)]
    d_epochs = [torch.full((n,), e, device=dev, dtype=torch.float64) for e in epochs]
    torch.cuda.synchronize()

    with torch.cuda.stream(stream):
        # per row: the first failing step and its status (later steps of a
        # failed row see its NaN output as invalid input)
        first_code = torch.zeros(n, device=dev, dtype=torch.int32)
        first_step = torch.full((n,), -1, device=dev, dtype=torch.int32)

    def step(k, src, dst):
        ctx.propagate_final_device(src.data_ptr(), d_epochs[k].data_ptr(), d_tf.data_ptr(), dst.data_ptr(),
                                   d_status.data_ptr(), d_steps.data_ptr(), d_evals.data_ptr(), n=n,
                                   d_ballistic=d_bal.data_ptr())
        with torch.cuda.stream(stream):
            new = (first_code == 0) & (d_status != 0)
            first_code.copy_(torch.where(new, d_status, first_code))
            first_step.copy_(torch.where(new, torch.full_like(first_step, k), first_step))

    # warm-up (also advances the batch)
    src, dst = d_a, d_b
    for k in range(args.warmup):
        step(k, src, dst)
        src, dst = dst, src
    stream.synchronize()

    # timed, device-resident
    events = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        evals_acc = torch.zeros((), device=dev, dtype=torch.int64)
    with ClockSampler(local) as clocks:
        e_start = torch.cuda.Event(enable_timing=True)
        e_end = torch.cuda.Event(enable_timing=True)
        e_start.record(stream)
        for k in range(args.warmup, args.warmup + args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()  # L2 flush between timed steps (256 MiB write)
            k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            k0.record(stream)
            step(k, src, dst)
            k1.record(stream)
            with torch.cuda.stream(stream):
                evals_acc += d_evals.sum()  # the device's per-trajectory counters of this step
            events.append((k0, k1))
            src, dst = dst, src
        e_end.record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    elapsed_ms = e_start.elapsed_time(e_end)
    # kernel attribution: the same K steps again (continuing the arc) with a
    # CUDA event on each side of every kernel launch; kept out of the pass
    # above because the events cost about 8% of the step time
    ctx.profile(True)
    with torch.cuda.stream(stream):
        prof_evals = torch.zeros((), device=dev, dtype=torch.int64)
    for k in range(args.warmup + args.steps, args.warmup + 2 * args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        step(k, src, dst)
        with torch.cuda.stream(stream):
            prof_evals += d_evals.sum()
        src, dst = dst, src
    stream.synchronize()
    ktimes = ctx.profile_read()
    ctx.profile(False)
    prof_evals = int(prof_evals.item())
    kernel_ms = [a.elapsed_time(b) for a, b in events]
    status_last = d_status.cpu().numpy()
    total_evals = int(evals_acc.item())

    t_max, total_all = combine_ranks(elapsed_ms, total_evals, world, dev)
    value = total_all / (t_max * 1e-3)

    # e2e: pinned host buffers through the host-buffer C ABI call
    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype).pin_memory().numpy()

    h_in = pinned((n, 6), torch.float64)
    h_in[:] = states
    h_out = pinned((n, 6), torch.float64)
    h_bal = pinned((n, 2), torch.float64)
    h_bal[:] = bal
    h_tf = pinned((n,), torch.float64)
    h_tf[:] = seg
    h_ep = pinned((n,), torch.float64)
    h_st = pinned((n,), torch.int32)
    h_steps = pinned((n,), torch.int64)
    h_evals = pinned((n,), torch.int64)
    for k in range(args.warmup):
        h_ep[:] = epochs[k]
        ctx.propagate_final(h_in, h_ep, h_tf, ballistic=h_bal, out=h_out, status=h_st, steps=h_steps,
                            evals=h_evals)
        h_in[:] = h_out
    if world > 1:
        dist.barrier()
    e2e_evals = 0
    t0 = time.perf_counter()
    for k in range(args.warmup, args.warmup + args.steps):
        h_ep[:] = epochs[k]
        ctx.propagate_final(h_in, h_ep, h_tf, ballistic=h_bal, out=h_out, status=h_st, steps=h_steps,
                            evals=h_evals)
        e2e_evals += int(h_evals.sum())
        h_in[:] = h_out
    e2e_s, e2e_evals = combine_ranks(time.perf_counter() - t0, e2e_evals, world, dev)
    e2e_value = e2e_evals / e2e_s
    h2d = n * 6 * 8 + n * 8 * 2 + n * 16
    d2h = n * 6 * 8 + n * 4 + n * 8 * 2

    line = None
    if rank == 0:
        peak = fp64_peak_tflops(torch, dev)
        fN = f_of_n(ORDER)
        # dominant kernel: the gravity stage; every force evaluation is one
        # gravity evaluation, F(70) algorithmic flops each
        dom = "persistent" if args.engine == "persistent" else "gravity"
        dom_ms, dom_launches = ktimes[dom]
        achieved = prof_evals * fN / (dom_ms * 1e-3) / 1e12
        step_tflops = total_evals * fN / (t_max * 1e-3) / 1e12
        kernel_shares = {k: {"ms": round(v[0], 3), "launches": v[1], "share": round(v[0] / max(1e-9, sum(
            x[0] for x in ktimes.values())), 4)} for k, v in ktimes.items() if v[1]}
        # kernels of the K profiled steps (plus one init kernel per step),
        # the same launch sequence as the timed steps
        launches = sum(v[1] for v in ktimes.values()) + (args.steps if args.engine == "pipeline" else 0)
        cpu = None
        if not args.no_cpu and world >= 1:
            threads = os.cpu_count() or 1
            v, dt, ev, ok = cpu_reference(args.cpu_sample, threads, method=args.method, eps=args.eps,
                                          segment_s=args.segment, atm_model=args.atm_model, srp=args.srp,
                                          frame=args.frame)
            cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"{args.cpu_sample} trajectories x one 5400 s segment ({ev} evals, {dt:.1f} s)"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(args),
            "engine": args.engine,
            "evals_per_step": total_evals / args.steps,
            "trajectory_days_per_s": world * n * seg / 86400.0 / (t_max * 1e-3 / args.steps),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": traffic_per_launch(dom, n),
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (no FP64 figure in "
                                        "MEASURED_PEAKS.json)",
                         "flops_per_eval": fN,
                         "kernel": "pl_gravity<4>" if dom == "gravity" else f"k_propagate<{args.method.upper()}>",
                         "kernel_ms": dom_ms, "kernel_launches": dom_launches,
                         "kernel_timing": "second pass of the K steps with a CUDA event on each side of "
                                          "every launch",
                         "whole_step_tflops": step_tflops, "whole_step_frac": step_tflops / peak,
                         "kernels": kernel_shares},
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "gpu_launches": launches,
            "status_ok_fraction": float((status_last == 0).mean()),
        }
        fc, fs = first_code.cpu().numpy(), first_step.cpu().numpy()
        if (fc != 0).any():
            bad = np.flatnonzero(fc)
            line["failures"] = {"first_status_counts": {str(c): int((fc == c).sum()) for c in np.unique(fc[bad])},
                                "rows": [[int(i), int(fs[i]), int(fc[i])] for i in bad[:16]]}
        if not args.no_forms and world == 1 and args.segment == SEGMENT_S and args.method == "dop853" \
                and args.eps == EPS and not args.split_degree and args.engine == "pipeline" and args.atm_model == 4 \
                and not args.srp and args.frame == "gmst":
            plain = {"force_evals_per_s": value, "trajectory_days_per_s": line["trajectory_days_per_s"]}
            line["forms"] = run_forms(args, text, states, bal, epoch, dev, plain)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return line


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
