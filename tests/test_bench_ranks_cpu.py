"""The multi-rank path of bench.py on CPU: two gloo ranks (one process each,
as torchrun starts them) combine their timings as the max over ranks and
their evaluation counts as the sum; each rank propagates its own seeded
trajectories (weak scaling, no data-path collective); under the reference arm
only rank 0 works."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import torch
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t, ev = bench.combine_ranks(10.0 + 5.0 * rank, 1000 * (rank + 1), world, torch.device("cpu"))
        e2e_t, e2e_ev = bench.combine_ranks(0.5 * (world - rank), 7 + rank, world, torch.device("cpu"))
        out.put((rank, t, ev, e2e_t, e2e_ev))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_max_time_and_summed_evaluations():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 2000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, t, ev, e2e_t, e2e_ev in got:
        assert (t, ev) == (15.0, 3000.0)  # max(10, 15), 1000 + 2000
        assert (e2e_t, e2e_ev) == (1.0, 15.0)


def test_one_rank_passes_its_own_figures():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.combine_ranks(12.5, 42, 1, None) == (12.5, 42.0)


def test_ranks_propagate_their_own_trajectories():
    sys.path.insert(0, str(ROOT))
    import bench

    _, s0, b0, _ = bench.make_workload(64, seed=0)
    _, s1, b1, _ = bench.make_workload(64, seed=1)
    assert not np.allclose(s0, s1) and not np.allclose(b0, b1)


def test_reference_arm_works_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("RANK", "1")
    called = []
    monkeypatch.setattr(bench, "cpu_reference", lambda *a, **k: called.append(a) or (1.0, 1.0, 1, 1))
    args = bench.parse(["--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"])
    assert bench.run_reference(args) is None
    assert not called and capsys.readouterr().out == ""


def test_reference_arm_runs_only_the_oracle():
    # the reference arm times the CPU restatement alone: the product's native
    # library must not be loaded by that process, and its config is the GPU
    # arm's config (its sample in a key of its own)
    import json
    import subprocess

    code = (
        "import sys, json; sys.path.insert(0, %r); import bench\n"
        "args = bench.parse(['--impl', 'reference', '--steps', '1', '--warmup', '0', '--cpu-sample', '2',"
        " '--segment', '120'])\n"
        "bench.run_reference(args)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'native_loaded': 'libbqp_b200' in maps, 'oracle_loaded': 'libprop_oracle' in maps,"
        " 'config': bench.bench_config(args)}))\n" % str(ROOT))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr
    lines = [json.loads(x) for x in r.stdout.strip().splitlines()]
    line, probe = lines[0], lines[1]
    assert not probe["native_loaded"] and probe["oracle_loaded"]
    assert line["impl"] == "reference" and line["config"] == probe["config"]
    assert line["sample"]["trajectories"] == 2 and line["value"] > 0
