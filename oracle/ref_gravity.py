"""ctypes wrapper of oracle/_ref/libref_gravity.so: the reference's own CUDA
gravity kernel (satpy_core/kernels/cuda/gravity.cu) behind the launcher in
ref_gravity_harness.cu.  TEST INFRASTRUCTURE ONLY, like the rest of oracle/:
the product never loads it."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libref_gravity.so"
_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(str(LIB_PATH))
        L.refgrav_scratch_doubles_per_state.restype = C.c_int64
        L.refgrav_launch.restype = C.c_int
        L.refgrav_launch.argtypes = [C.c_int64, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def scratch_doubles_per_state() -> int:
    return int(lib().refgrav_scratch_doubles_per_state())


def launch(n, d_states6, d_rot9, order, stride, d_c, d_s, d_acc3, d_scratch, stream) -> None:
    """All pointers are device addresses (ints); enqueued on `stream`."""
    rc = lib().refgrav_launch(int(n), d_states6, d_rot9, int(order), int(stride), d_c, d_s, d_acc3, d_scratch,
                              stream)
    if rc != 0:
        raise RuntimeError(f"reference gravity kernel launch failed: cudaError {rc}")
