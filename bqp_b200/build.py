"""Build libbqp_b200.so in-tree with nvcc for sm_100a.

    python -m bqp_b200.build [--verbose]

The shared library lands in ``bqp_b200/_lib/`` and is what the Python layer
loads; nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "_lib"
LIB = LIB_DIR / "libbqp_b200.so"
SOURCES = ["propagate.cu", "pipeline.cu", "eclipse.cu", "sigma.cu", "mlp.cu", "surrogate.cu", "space_weather.cu", "ephemeris.cu",
           "bqp_api.cu", "frame_time.cpp"]
HEADERS = ["kernels.cuh", "gravity.cuh", "gravity_cta.cuh", "jb2008.cuh", "physics.cuh", "launch.h", "rk_tableaus.h",
           "traj.cuh", "eclipse.cuh", "tc_gemm.cuh", "space_weather.h", "ephemeris.h", "surrogate.h",
           "frame_time.h", "frame_time_host.h", "iau2000a_tables.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [PKG.parent / "include" / "bqp_prop.h"]
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    LIB_DIR.mkdir(exist_ok=True)
    objs = []
    flags = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", *ARCH,
             "-I", str(CSRC), "-I", str(PKG.parent / "include")]
    # extra nvcc definitions for measured build variants (e.g. -DBQP_DRAG_MIN_BLOCKS=4)
    flags += os.environ.get("BQP_NVCC_DEFINES", "").split()
    if verbose:
        flags += ["-Xptxas", "-v"]
    for src in SOURCES:
        obj = LIB_DIR / (Path(src).stem + ".o")
        cmd = [nvcc(), *flags, "-c", str(CSRC / src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr, file=sys.stderr)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "--cudart", "static", "-o", str(tmp), *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose="--verbose" in sys.argv))
