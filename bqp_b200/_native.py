"""ctypes binding of libbqp_b200.so (the C ABI in include/bqp_prop.h).

The library is built in-tree (``python -m bqp_b200.build``).  Loading fails
loudly when it is missing: there is no CPU fallback for the propagator.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from pathlib import Path

import numpy as np

from . import build as _build

LIB_PATH = _build.LIB

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)
_fp = C.POINTER(C.c_float)
_vp = C.c_void_p

# per-trajectory status codes (BQP_ST_*)
STATUS_NAMES = {
    0: "ok", 1: "max_steps_exceeded", 2: "step_underflow", 3: "invalid_input",
    4: "non_finite_state", 5: "max_rejects_exceeded", 6: "gravity_invalidradius",
    7: "rebase_failed", 8: "restart_budget_exhausted", 9: "ground", 10: "watchdog",
    # the reference's eclipse_error_name (eclipse_coordinator.rs:950-966)
    11: "eclipse_envelope", 12: "eclipse_chatter", 13: "eclipse_bracket", 14: "eclipse_non_progress",
    15: "eclipse_geometry", 16: "eclipse_split_limit",
    # GravityError::InvalidTime from the IAU frame authority
    17: "frame_invalid_time",
}
ST_ECLIPSE_ENVELOPE = 11
ECLIPSE_STATUSES = frozenset(range(11, 17))
ST_OK, ST_GROUND, ST_GRAVITY_RADIUS = 0, 9, 6
ST_FRAME_TIME = 17
FRAMES = {"gmst": 0, "iau2006": 1}  # BQP_FRAME_*

FORCE_DRAG, FORCE_SRP, FORCE_SUN, FORCE_MOON = 1, 2, 4, 8
METHODS = {"dopri5_solver": 0, "dop853": 1, "dopri5": 2, "vern7": 3, "vern9": 4}
ENGINES = {"pipeline": 0, "persistent": 1}

E_ARG, E_CUDA, E_COEFF, E_UNSUPPORTED, E_NOMEM = -1, -2, -3, -4, -5
NOALLOC_MAX_TRAJ = 16384  # BQP_NOALLOC_MAX_TRAJ
KERNEL_CLASSES = ("prep", "gravity", "drag", "control", "persistent")  # BQP_KCLASS_*
SURROGATE_PARAMS = 199427  # BQP_SURROGATE_PARAMS
SURROGATE_DEGREE = 8  # BQP_SURROGATE_DEGREE


class ForceConfig(C.Structure):
    """Mirror of ``bqp_force_config``."""
    _fields_ = [
        ("order", C.c_int32), ("force_flags", C.c_int32), ("atm_model", C.c_int32),
        ("method", C.c_int32), ("error_control", C.c_int32), ("ground_check", C.c_int32),
        ("eps", C.c_double), ("rtol", C.c_double), ("atol", C.c_double), ("dt_max", C.c_double),
        ("am_ratio", C.c_double), ("cd", C.c_double), ("earth_radius", C.c_double),
        ("omega_earth", C.c_double), ("mu_sun", C.c_double), ("mu_moon", C.c_double),
        ("jb_drivers", C.c_double * 9), ("max_steps", C.c_int64), ("max_attempts", C.c_int64),
        ("max_kernel_seconds", C.c_double), ("engine", C.c_int32), ("gravity_threads", C.c_int32),
        ("gravity_slots", C.c_int32), ("drag_quadrature", C.c_int32), ("split_degree", C.c_int32),
        ("drag_fp32", C.c_int32), ("surrogate", C.c_int32), ("surrogate_check", C.c_double),
        ("cr", C.c_double), ("p_sun", C.c_double),
    ]


class NativeError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()

# (name, restype, argtypes) of every exported symbol of include/bqp_prop.h
SIGNATURES = [
    ("bqp_force_config_default", None, [C.POINTER(ForceConfig)]),
    ("bqp_last_error", C.c_char_p, []),
    ("bqp_ctx_create", C.c_int, [C.c_char_p, C.c_int64, C.POINTER(ForceConfig), C.POINTER(_vp)]),
    ("bqp_ctx_destroy", C.c_int, [_vp]),
    ("bqp_ctx_set_stream", C.c_int, [_vp, _vp]),
    ("bqp_ctx_info", C.c_int, [_vp, _lp]),
    ("bqp_ctx_set_config", C.c_int, [_vp, C.POINTER(ForceConfig)]),
    ("bqp_ctx_info_fit", C.c_int, [_vp, _dp]),
    ("bqp_jb_fit_check", C.c_int, [_dp, _dp]),
    ("bqp_jb_density", C.c_int, [C.c_int32, C.c_int32, C.c_int64, _dp, _dp]),
    ("bqp_ecl_scan_check", C.c_int, [_vp, C.c_int64, _dp, C.c_int32, _dp]),
    ("bqp_utc_jd", C.c_int, [C.c_int64, _dp, _dp, _dp]),
    ("bqp_ctx_set_jb_drivers", C.c_int, [_vp, C.c_char_p, C.c_int64, C.c_char_p, C.c_int64, C.c_double,
                                         C.c_double]),
    ("bqp_ctx_jb_lookup", C.c_int, [_vp, _dp, C.c_int64, _dp, _ip]),
    ("bqp_ctx_set_ephemeris", C.c_int, [_vp, C.c_int32, C.c_char_p, C.c_int64]),
    ("bqp_ctx_body_positions", C.c_int, [_vp, C.c_int32, _dp, C.c_int64, _dp]),
    ("bqp_ephemeris_check", C.c_int, [C.c_int32, C.c_char_p, C.c_int64, _dp, C.c_int64, _dp, _lp]),
    ("bqp_jb_drivers_check", C.c_int, [C.c_char_p, C.c_int64, C.c_char_p, C.c_int64, _dp, C.c_int64, _dp, _ip,
                                       _lp]),
    ("bqp_ctx_profile", C.c_int, [_vp, C.c_int32]),
    ("bqp_ctx_profile_read", C.c_int, [_vp, _dp, _lp]),
    ("bqp_gravity_eval", C.c_int, [_vp, C.c_int64, _dp, _dp, _ip]),
    ("bqp_gravity_eval_device", C.c_int, [_vp, C.c_int64, _vp, _vp, _vp]),
    ("bqp_rhs_eval", C.c_int, [_vp, C.c_int64, _dp, _dp, _dp, _dp, _dp, _dp, _dp]),
    ("bqp_rhs_eval_device", C.c_int, [_vp, C.c_int64, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("bqp_propagate_final", C.c_int, [_vp, C.c_int64, _dp, C.c_int32, _dp, C.c_double, _dp, _dp, _dp,
                                      _ip, _lp, _lp]),
    ("bqp_propagate_final_device", C.c_int, [_vp, C.c_int64, _vp, C.c_int32, _vp, C.c_double, _vp, _vp,
                                             _vp, _vp, _vp, _vp]),
    ("bqp_propagate_final_noalloc", C.c_int, [_vp, C.c_int64, _dp, C.c_int32, _dp, C.c_double, _dp, _dp,
                                              _dp, _ip, _lp, _lp]),
    ("bqp_propagate_sampled", C.c_int, [_vp, C.c_int64, _dp, C.c_int32, _dp, C.c_double, _dp, C.c_int32,
                                        _dp, C.c_int32, _dp, _ip, _lp, _lp]),
    ("bqp_propagate_sampled_device", C.c_int, [_vp, C.c_int64, _vp, C.c_int32, _vp, C.c_double, _vp,
                                               C.c_int32, _vp, C.c_int32, _vp, _vp, _vp, _vp]),
    ("bqp_sigma_propagate", C.c_int, [_vp, C.c_int64, _dp, _dp, C.c_int32, C.c_double, C.c_double, C.c_double,
                                      _dp, C.c_double, _dp, _dp, _dp, _dp, _ip, _lp]),
    ("bqp_sigma_propagate_device", C.c_int, [_vp, C.c_int64, _vp, _vp, C.c_int32, C.c_double, C.c_double,
                                             C.c_double, _vp, C.c_double, _vp, _vp, _vp, _vp, _vp, _vp]),
    ("bqp_sigma_weights", C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_double, _ip, _dp, _dp, _dp]),
    ("bqp_gemm_bf16_device", C.c_int, [C.c_int64, C.c_int64, C.c_int64, _vp, _vp, _vp, _vp]),
    ("bqp_surrogate_train", C.c_int, [_vp, C.c_int64, C.c_int32, C.c_int32, C.c_double, C.c_uint64, _dp]),
    ("bqp_surrogate_infer", C.c_int, [_vp, C.c_int64, _dp, _dp, C.c_int32]),
    ("bqp_surrogate_infer_device", C.c_int, [_vp, C.c_int64, _vp, _vp, C.c_int32]),
    ("bqp_surrogate_params", C.c_int, [_vp, _fp, _dp]),
    ("bqp_surrogate_set_params", C.c_int, [_vp, _fp, C.c_double]),
    ("bqp_surrogate_grad", C.c_int, [_vp, C.c_int32, _fp, _fp, _fp, _fp, _dp, _fp]),
    ("bqp_eci_to_equinoctial", C.c_int, [C.c_int64, _dp, _dp, _ip]),
    ("bqp_equinoctial_to_eci", C.c_int, [C.c_int64, _dp, _dp, _dp]),
    ("bqp_kep_to_eci", C.c_int, [C.c_int64, _dp, _dp]),
    ("bqp_eci_to_kep", C.c_int, [C.c_int64, _dp, _dp]),
    ("bqp_ctx_set_frame", C.c_int, [_vp, C.c_int32, _dp, C.c_int32, C.c_int32]),
    ("bqp_ctx_set_frame_span", C.c_int, [_vp, C.c_double, C.c_double]),
    ("bqp_frame_nut", None, [C.c_double, C.c_double, C.c_int32, _dp]),
    ("bqp_frame_obl06", C.c_double, [C.c_double, C.c_double]),
    ("bqp_frame_pfw06", None, [C.c_double, C.c_double, _dp]),
    ("bqp_frame_xys06a", None, [C.c_double, C.c_double, _dp]),
    ("bqp_frame_c2ixys", None, [C.c_double, C.c_double, C.c_double, _dp]),
    ("bqp_frame_sp00", C.c_double, [C.c_double, C.c_double]),
    ("bqp_frame_pom00", None, [C.c_double, C.c_double, C.c_double, _dp]),
    ("bqp_frame_era", C.c_double, [C.c_double, C.c_double]),
    ("bqp_frame_utc_calendar", C.c_int, [C.c_int32] * 5 + [C.c_double, _dp]),
    ("bqp_frame_tai_seconds", C.c_int, [C.c_int64, _dp, _dp, _dp]),
    ("bqp_frame_matrix", C.c_int, [C.c_int32] * 5 + [C.c_double, C.c_int32, C.c_double, _dp, C.c_int32,
                                                      C.c_int32, _dp]),
    ("bqp_frame_derivatives", C.c_int, [C.c_int32] * 5 + [C.c_double, C.c_int32, C.c_double, _dp, C.c_int32,
                                                           C.c_int32, _dp, _dp, _dp]),
    ("bqp_frame_eop_from_finals", C.c_int64, [C.c_char_p, C.c_int64, C.c_int64, _ip, _dp]),
    ("bqp_frame_transform_state", C.c_int, [C.c_int32] * 5 + [C.c_double, C.c_int32, C.c_double, _dp, C.c_int32,
                                                               C.c_int32, _dp, _dp, _dp, _dp, _dp, _dp]),
    ("bqp_frame_authority_new", _vp, [_dp, C.c_int32, C.c_int32]),
    ("bqp_frame_authority_free", None, [_vp]),
    ("bqp_frame_authority_intervals", C.c_int, [_vp, _dp]),
    ("bqp_frame_authority_rotation", C.c_int, [_vp, C.c_int64, _dp, _dp, _dp]),
    ("bqp_frame_authority_segments", C.c_int64, [_vp, C.c_double, C.c_double, C.c_int64, _lp, _dp]),
]


def lib():
    """Load (building first if stale) the native library."""
    global _lib
    with _lock:
        if _lib is None:
            try:
                _build.build()
            except Exception as exc:  # no nvcc here: use the shipped build if present
                if not LIB_PATH.exists():
                    raise ImportError(f"libbqp_b200.so is missing and could not be built: {exc}")
            if not LIB_PATH.exists():
                raise ImportError(f"libbqp_b200.so not found at {LIB_PATH}")
            L = C.CDLL(str(LIB_PATH))
            for name, res, args in SIGNATURES:
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def last_error() -> str:
    return lib().bqp_last_error().decode()


def check(rc: int) -> None:
    if rc != 0:
        raise NativeError(rc, last_error())


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def lptr(a: np.ndarray):
    return a.ctypes.data_as(_lp)


def f64(a, shape=None) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        out = out.reshape(shape)
    return out


def default_config() -> ForceConfig:
    cfg = ForceConfig()
    lib().bqp_force_config_default(C.byref(cfg))
    return cfg


class Context:
    """Owns one native propagator context (device field table + settings)."""

    def __init__(self, coeff_text: str, cfg: ForceConfig):
        self._h = _vp()
        raw = coeff_text.encode()
        check(lib().bqp_ctx_create(raw, len(raw), C.byref(cfg), C.byref(self._h)))
        self.cfg = cfg

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().bqp_ctx_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        out = np.zeros(4, dtype=np.int64)
        check(lib().bqp_ctx_info(self._h, lptr(out)))
        w = C.c_double(0.0)
        check(lib().bqp_ctx_info_fit(self._h, C.byref(w)))
        return {"order": int(out[0]), "cells": int(out[1]), "table_bytes": int(out[2]),
                "table_in_shared_memory": bool(out[3]), "jb_fit_worst_rel": w.value}

    def set_config(self, cfg: ForceConfig):
        check(lib().bqp_ctx_set_config(self._h, C.byref(cfg)))
        self.cfg = cfg

    def profile(self, on: bool = True):
        """Start (clearing the totals) or stop kernel timing by class."""
        check(lib().bqp_ctx_profile(self._h, int(bool(on))))

    def profile_read(self):
        """{class: (ms, launches)} since profiling was switched on."""
        ms = np.zeros(len(KERNEL_CLASSES))
        n = np.zeros(len(KERNEL_CLASSES), dtype=np.int64)
        check(lib().bqp_ctx_profile_read(self._h, dptr(ms), lptr(n)))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(KERNEL_CLASSES)}

    def set_jb_drivers(self, solfsmy, dtcfile, span_jd=(0.0, 0.0)):
        """Take the JB2008 drivers per evaluation from SET space-weather files
        (SOLFSMY and DTCFILE: text, bytes or a path; both None: back to the
        configured fixed drivers).  span_jd = the UTC Julian days the
        propagations will cover, which bounds the drag sweep fits ((0, 0):
        the whole table).  ValueError names the first rejected line."""
        if solfsmy is None and dtcfile is None:
            check(lib().bqp_ctx_set_jb_drivers(self._h, None, 0, None, 0, 0.0, 0.0))
            return
        sol, dtc = _text_bytes(solfsmy), _text_bytes(dtcfile)
        rc = lib().bqp_ctx_set_jb_drivers(self._h, sol, len(sol), dtc, len(dtc), float(span_jd[0]),
                                          float(span_jd[1]))
        if rc == E_ARG:
            raise ValueError(last_error())
        check(rc)

    def set_frame(self, frame: str = "gmst", eop=None, first_mjd: int = 41684):
        """Earth-fixed frame of gravity and drag: "gmst" (the z-rotation by
        GMST) or "iau2006" (GCRS->ITRS of the IAU 2006/2000A chain from 1800 s
        segments).  eop: [n][5] records per UTC day from first_mjd (x_p, y_p
        arcsec, UT1-UTC s, dX, dY mas; the reference's eop_table.bin as an
        array), None for zero EOP."""
        mode = FRAMES[frame]
        if eop is None:
            rc = lib().bqp_ctx_set_frame(self._h, mode, None, 0, 0)
        else:
            e = f64(eop).reshape(-1, 5)
            rc = lib().bqp_ctx_set_frame(self._h, mode, dptr(e), int(first_mjd), e.shape[0])
        if rc == E_ARG:
            raise ValueError(last_error())
        check(rc)

    def set_frame_span(self, jd_lo=0.0, jd_hi=0.0):
        """Segments of the IAU frame for UTC days [jd_lo, jd_hi], built once;
        calls then skip the per-call epoch readback.  (0, 0): per call."""
        rc = lib().bqp_ctx_set_frame_span(self._h, float(jd_lo), float(jd_hi))
        if rc == E_ARG:
            raise ValueError(last_error())
        check(rc)

    def set_ephemeris(self, body: str, catalogue):
        """Take the Sun's or the Moon's position from a precomputed "DUST"
        catalogue (bytes or a path; None: back to the analytic series).
        ValueError names what the loader rejected."""
        b = BODIES[body]
        if catalogue is None:
            check(lib().bqp_ctx_set_ephemeris(self._h, b, None, 0))
            return
        data = _file_bytes(catalogue)
        rc = lib().bqp_ctx_set_ephemeris(self._h, b, data, len(data))
        if rc == E_ARG:
            raise ValueError(last_error())
        check(rc)

    def body_positions(self, body: str, utc_jd):
        """[n, 3] km: the body's positions as the force kernels take them."""
        jd = f64(np.atleast_1d(utc_jd))
        out = np.empty((jd.size, 3))
        check(lib().bqp_ctx_body_positions(self._h, BODIES[body], dptr(jd), jd.size, dptr(out)))
        return out

    def jb_lookup(self, utc_jd):
        """(drivers [n, 9]: F10, F81c, S10, S81c, M10, M81c, Y10, Y81c, dTc,
        NaN rows where the tables do not cover the instant; ok [n] bool),
        evaluated by the device lookup the force kernels use."""
        jd = f64(np.atleast_1d(utc_jd))
        out = np.empty((jd.size, 9))
        ok = np.empty(jd.size, dtype=np.int32)
        check(lib().bqp_ctx_jb_lookup(self._h, dptr(jd), jd.size, dptr(out), iptr(ok)))
        return out, ok.astype(bool)

    def set_stream(self, stream_ptr: int):
        check(lib().bqp_ctx_set_stream(self._h, _vp(stream_ptr)))

    # ---------------------------------------------------------------- host
    def gravity(self, pos_km):
        p = f64(pos_km).reshape(-1, 3)
        acc = np.empty_like(p)
        st = np.empty(p.shape[0], dtype=np.int32)
        check(lib().bqp_gravity_eval(self._h, p.shape[0], dptr(p), dptr(acc), iptr(st)))
        return acc, st

    def rhs(self, equ, seg_t0, epoch_jd, t, delta, ballistic=None):
        equ = f64(equ).reshape(-1, 6)
        n = equ.shape[0]
        seg_t0 = f64(np.broadcast_to(seg_t0, (n,)))
        epoch_jd = f64(np.broadcast_to(epoch_jd, (n,)))
        t = f64(np.broadcast_to(t, (n,)))
        delta = f64(delta).reshape(n, 6)
        bal = None if ballistic is None else f64(np.broadcast_to(ballistic, (n, 2)))
        out = np.empty((n, 6))
        check(lib().bqp_rhs_eval(self._h, n, dptr(equ), dptr(seg_t0), dptr(epoch_jd), dptr(t), dptr(delta),
                                 None if bal is None else dptr(bal), dptr(out)))
        return out

    def propagate_final(self, states, epoch_jd, tf, t0=0.0, ballistic=None, equinoctial=False, out=None,
                        status=None, steps=None, evals=None):
        """Host-buffer call; `out`/`status`/`steps`/`evals` may be preallocated
        (e.g. pinned) arrays of the right dtype and shape."""
        s = f64(states).reshape(-1, 6)
        n = s.shape[0]
        ep = f64(np.broadcast_to(epoch_jd, (n,)))
        tfa = f64(np.broadcast_to(tf, (n,)))
        bal = None if ballistic is None else f64(np.broadcast_to(ballistic, (n, 2)))
        out = np.empty((n, 6)) if out is None else out
        st = np.empty(n, dtype=np.int32) if status is None else status
        steps = np.empty(n, dtype=np.int64) if steps is None else steps
        evals = np.empty(n, dtype=np.int64) if evals is None else evals
        assert out.shape == (n, 6) and out.dtype == np.float64 and out.flags.c_contiguous
        assert st.dtype == np.int32 and steps.dtype == np.int64 and evals.dtype == np.int64
        check(lib().bqp_propagate_final(self._h, n, dptr(s), int(equinoctial), dptr(ep), float(t0), dptr(tfa),
                                        None if bal is None else dptr(bal), dptr(out), iptr(st), lptr(steps),
                                        lptr(evals)))
        return out, st, steps, evals

    def propagate_final_noalloc(self, states, epoch_jd, tf, t0=0.0, ballistic=None, equinoctial=False):
        """Like propagate_final, through the entry point that allocates no
        device memory (at most NOALLOC_MAX_TRAJ rows; persistent kernel)."""
        s = f64(states).reshape(-1, 6)
        n = s.shape[0]
        ep = f64(np.broadcast_to(epoch_jd, (n,)))
        tfa = f64(np.broadcast_to(tf, (n,)))
        bal = None if ballistic is None else f64(np.broadcast_to(ballistic, (n, 2)))
        out = np.empty((n, 6))
        st = np.empty(n, dtype=np.int32)
        steps = np.empty(n, dtype=np.int64)
        evals = np.empty(n, dtype=np.int64)
        check(lib().bqp_propagate_final_noalloc(self._h, n, dptr(s), int(equinoctial), dptr(ep), float(t0),
                                                dptr(tfa), None if bal is None else dptr(bal), dptr(out),
                                                iptr(st), lptr(steps), lptr(evals)))
        return out, st, steps, evals

    def propagate_sampled(self, states, epoch_jd, tf, t_eval, t0=0.0, deltas=False, equinoctial=False):
        s = f64(states).reshape(-1, 6)
        n = s.shape[0]
        ep = f64(np.broadcast_to(epoch_jd, (n,)))
        tfa = f64(np.broadcast_to(tf, (n,)))
        te = f64(t_eval).reshape(-1)
        out = np.empty((n, te.size, 6))
        st = np.empty(n, dtype=np.int32)
        steps = np.empty(n, dtype=np.int64)
        evals = np.empty(n, dtype=np.int64)
        check(lib().bqp_propagate_sampled(self._h, n, dptr(s), int(equinoctial), dptr(ep), float(t0), dptr(tfa),
                                          te.size, dptr(te), int(deltas), dptr(out), iptr(st), lptr(steps),
                                          lptr(evals)))
        return out, st, steps, evals

    def sigma_propagate(self, mean, cov, epoch_jd, tf, sigma_set="julier7", alpha=1e-3, beta=2.0, kappa=0.0,
                        t0=0.0, ballistic=None):
        """Unscented propagation of (mean[n][6], cov[n][6][6]) to tf[n]:
        returns mean_out, cov_out, status, evals."""
        m = f64(mean).reshape(-1, 6)
        n = m.shape[0]
        c = f64(cov).reshape(n, 36)
        ep = f64(np.broadcast_to(epoch_jd, (n,)))
        tfa = f64(np.broadcast_to(tf, (n,)))
        bal = None if ballistic is None else f64(np.broadcast_to(ballistic, (n, 2)))
        mo = np.empty((n, 6))
        co = np.empty((n, 36))
        st = np.empty(n, dtype=np.int32)
        ev = np.empty(n, dtype=np.int64)
        check(lib().bqp_sigma_propagate(self._h, n, dptr(m), dptr(c), SIGMA_SETS[sigma_set], alpha, beta, kappa,
                                        dptr(ep), float(t0), dptr(tfa), None if bal is None else dptr(bal),
                                        dptr(mo), dptr(co), iptr(st), lptr(ev)))
        return mo, co.reshape(n, 6, 6), st, ev

    # ------------------------------------------------------------ surrogate
    def surrogate_train(self, samples=1 << 20, epochs=4, batch=8192, lr=2e-3, seed=1):
        """Train the degree > 8 gravity surrogate on the GPU; returns the
        per-epoch training loss (normalised MSE)."""
        loss = np.zeros(epochs)
        check(lib().bqp_surrogate_train(self._h, int(samples), int(epochs), int(batch), float(lr), int(seed),
                                        dptr(loss)))
        return loss

    def surrogate_infer(self, pos_km, add_low=True, fused=True):
        p = f64(pos_km).reshape(-1, 3)
        acc = np.empty_like(p)
        flags = (1 if add_low else 0) | (0 if fused else 2)
        check(lib().bqp_surrogate_infer(self._h, p.shape[0], dptr(p), dptr(acc), flags))
        return acc

    def surrogate_infer_device(self, n, d_pos, d_acc, add_low=True):
        check(lib().bqp_surrogate_infer_device(self._h, int(n), _vp(d_pos), _vp(d_acc), int(add_low)))

    def surrogate_params(self):
        params = np.zeros(SURROGATE_PARAMS, dtype=np.float32)
        sigma = C.c_double(0.0)
        check(lib().bqp_surrogate_params(self._h, params.ctypes.data_as(_fp), C.byref(sigma)))
        return params, sigma.value

    def surrogate_set_params(self, params, sigma):
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == SURROGATE_PARAMS
        check(lib().bqp_surrogate_set_params(self._h, p.ctypes.data_as(_fp), float(sigma)))

    def surrogate_grad(self, params, x, t):
        """(loss, grad[SURROGATE_PARAMS], y[B][3]) of one batch on the GPU."""
        p = np.ascontiguousarray(params, dtype=np.float32)
        xb = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 4)
        tb = np.ascontiguousarray(t, dtype=np.float32).reshape(-1, 3)
        g = np.zeros(SURROGATE_PARAMS, dtype=np.float32)
        y = np.zeros((xb.shape[0], 3), dtype=np.float32)
        loss = C.c_double(0.0)
        check(lib().bqp_surrogate_grad(self._h, xb.shape[0], p.ctypes.data_as(_fp), xb.ctypes.data_as(_fp),
                                       tb.ctypes.data_as(_fp), g.ctypes.data_as(_fp), C.byref(loss),
                                       y.ctypes.data_as(_fp)))
        return loss.value, g, y

    # -------------------------------------------------------------- device
    def propagate_final_device(self, d_in, d_epoch, d_tf, d_out, d_status, d_steps=None, d_evals=None,
                               n=None, t0=0.0, d_ballistic=None, equinoctial=False):
        """Device-pointer variant: arguments are raw CUDA addresses (ints)."""
        check(lib().bqp_propagate_final_device(self._h, int(n), _vp(d_in), int(equinoctial), _vp(d_epoch),
                                               float(t0), _vp(d_tf), _vp(d_ballistic) if d_ballistic else None,
                                               _vp(d_out), _vp(d_status), _vp(d_steps) if d_steps else None,
                                               _vp(d_evals) if d_evals else None))

    def ecl_scan(self, paths, warp=False):
        """The eclipse crossing scan on Hermite paths [n][16] (see
        bqp_ecl_scan_check): [n][7] status, found, sides, t_old, t_new, bound."""
        p = f64(paths).reshape(-1, 16)
        out = np.empty((p.shape[0], 7))
        check(lib().bqp_ecl_scan_check(self._h, p.shape[0], dptr(p), int(bool(warp)), dptr(out)))
        return out

    def gravity_device(self, n, d_pos, d_acc, d_status=None):
        check(lib().bqp_gravity_eval_device(self._h, int(n), _vp(d_pos), _vp(d_acc),
                                            _vp(d_status) if d_status else None))


# ----------------------------------------------------------- host helpers
SIGMA_SETS = {"julier7": 0, "merwe13": 1}  # BQP_SIGMA_*


def sigma_weights(sigma_set="julier7", alpha=1e-3, beta=2.0, kappa=0.0):
    """(points, wm, wc, offsets[7][6]) of a sigma set."""
    pts = C.c_int32(0)
    wm = np.zeros(13)
    wc = np.zeros(13)
    off = np.zeros((7, 6))
    check(lib().bqp_sigma_weights(SIGMA_SETS[sigma_set], alpha, beta, kappa, C.byref(pts), dptr(wm), dptr(wc),
                                  dptr(off)))
    p = pts.value
    return p, wm[:p].copy(), wc[:p].copy(), off


BODIES = {"sun": 0, "moon": 1}


def _file_bytes(x) -> bytes:
    """Binary file contents from bytes or a path."""
    if isinstance(x, (bytes, bytearray, memoryview)):
        return bytes(x)
    return open(x, "rb").read()


def ephemeris_check(body: str, catalogue, utc_jd=()):
    """Host-only parse of a "DUST" catalogue and positions at utc_jd:
    (sample count, positions [n, 3] km).  ValueError names what was rejected."""
    data = _file_bytes(catalogue)
    jd = f64(np.atleast_1d(np.asarray(utc_jd, dtype=np.float64)))
    out = np.empty((jd.size, 3))
    n = np.zeros(1, dtype=np.int64)
    rc = lib().bqp_ephemeris_check(BODIES[body], data, len(data), dptr(jd), jd.size, dptr(out), lptr(n))
    if rc == E_ARG:
        raise ValueError(last_error())
    check(rc)
    return int(n[0]), out


def _text_bytes(x) -> bytes:
    """File contents from text, bytes or a path."""
    if isinstance(x, bytes):
        return x
    if isinstance(x, os.PathLike) or (isinstance(x, str) and "\n" not in x and os.path.isfile(x)):
        return open(x, "rb").read()
    return str(x).encode()


def jb_drivers_check(solfsmy, dtcfile, utc_jd=()):
    """Host-only parse of SET space-weather files and lookups at utc_jd:
    ((SOLFSMY rows, DTCFILE rows), drivers [n, 9], ok [n] bool).  ValueError
    names the first rejected line."""
    sol, dtc = _text_bytes(solfsmy), _text_bytes(dtcfile)
    jd = f64(np.atleast_1d(np.asarray(utc_jd, dtype=np.float64)))
    out = np.empty((jd.size, 9))
    ok = np.empty(jd.size, dtype=np.int32)
    counts = np.zeros(2, dtype=np.int64)
    rc = lib().bqp_jb_drivers_check(sol, len(sol), dtc, len(dtc), dptr(jd), jd.size, dptr(out), iptr(ok),
                                    lptr(counts))
    if rc == E_ARG:
        raise ValueError(last_error())
    check(rc)
    return (int(counts[0]), int(counts[1])), out, ok.astype(bool)


def jb_density(model: int, inputs, fp32: bool = False) -> np.ndarray:
    """Host evaluation of the JB2008 density by the kernels' own function:
    inputs [n][14] (see bqp_jb_density), model 4-7; fp32: the split form's
    FP32 arithmetic (models 5-7)."""
    x = f64(inputs).reshape(-1, 14)
    out = np.empty(x.shape[0])
    check(lib().bqp_jb_density(int(model), int(bool(fp32)), x.shape[0], dptr(x), dptr(out)))
    return out


def utc_jd(jd0, t) -> np.ndarray:
    """UTC Julian days of instants t (elapsed seconds) after UTC epochs jd0,
    as the kernels form them (bqp_utc_jd)."""
    t = f64(np.atleast_1d(t))
    j = f64(np.broadcast_to(jd0, t.shape))
    out = np.empty(t.size)
    check(lib().bqp_utc_jd(t.size, dptr(j), dptr(t), dptr(out)))
    return out


def jb_fit_check(drivers=(150.0,) * 8 + (20.0,)):
    """Host-side build and self-check of the JB2008 sweep fits: dict of the
    worst relative errors and the 2-D fits' T_inf range."""
    w = np.zeros(6)
    check(lib().bqp_jb_fit_check(dptr(f64(drivers)), dptr(w)))
    return {"fixed": w[0], "mid": w[1], "uplow": w[2], "uphigh": w[3], "tinf_range": (w[4], w[5])}


def eci_to_equinoctial(eci):
    e = f64(eci).reshape(-1, 6)
    out = np.empty_like(e)
    ok = np.empty(e.shape[0], dtype=np.int32)
    check(lib().bqp_eci_to_equinoctial(e.shape[0], dptr(e), dptr(out), iptr(ok)))
    return out, ok.astype(bool)


def equinoctial_to_eci(equ, tof=0.0):
    e = f64(equ).reshape(-1, 6)
    t = f64(np.broadcast_to(tof, (e.shape[0],)))
    out = np.empty_like(e)
    check(lib().bqp_equinoctial_to_eci(e.shape[0], dptr(e), dptr(t), dptr(out)))
    return out


def kep_to_eci(kep):
    k = f64(kep).reshape(-1, 6)
    out = np.empty_like(k)
    check(lib().bqp_kep_to_eci(k.shape[0], dptr(k), dptr(out)))
    return out


def eci_to_kep(eci):
    e = f64(eci).reshape(-1, 6)
    out = np.empty_like(e)
    check(lib().bqp_eci_to_kep(e.shape[0], dptr(e), dptr(out)))
    return out


# ---------------------------------------------------------- IAU 2006/2000A
def frame_nut(d1, d2, iau2006=True):
    o = np.zeros(2)
    lib().bqp_frame_nut(float(d1), float(d2), int(bool(iau2006)), dptr(o))
    return o


def frame_obl06(d1, d2):
    return lib().bqp_frame_obl06(float(d1), float(d2))


def frame_pfw06(d1, d2):
    o = np.zeros(4)
    lib().bqp_frame_pfw06(float(d1), float(d2), dptr(o))
    return o


def frame_xys06a(d1, d2):
    o = np.zeros(3)
    lib().bqp_frame_xys06a(float(d1), float(d2), dptr(o))
    return o


def frame_c2ixys(x, y, s):
    o = np.zeros(9)
    lib().bqp_frame_c2ixys(float(x), float(y), float(s), dptr(o))
    return o.reshape(3, 3)


def frame_sp00(d1, d2):
    return lib().bqp_frame_sp00(float(d1), float(d2))


def frame_pom00(xp, yp, sp):
    o = np.zeros(9)
    lib().bqp_frame_pom00(float(xp), float(yp), float(sp), dptr(o))
    return o.reshape(3, 3)


def frame_era(u1, u2):
    return lib().bqp_frame_era(float(u1), float(u2))


def utc_calendar(y, m, d, hh=0, mm=0, ss=0.0):
    """Two-part UTC quasi-JD of a calendar instant (ERFA dtf2d "UTC")."""
    o = np.zeros(2)
    if lib().bqp_frame_utc_calendar(y, m, d, hh, mm, float(ss), dptr(o)) != 0:
        raise ValueError("invalid UTC calendar instant")
    return o[0], o[1]


def tai_seconds(utc_jd, utc_jd2=None):
    """Continuous TAI seconds (from 0h TAI of MJD 41684) of UTC Julian days,
    one part or two; NaN before 1972."""
    a = f64(np.atleast_1d(utc_jd))
    out = np.empty(a.size)
    b = None if utc_jd2 is None else f64(np.broadcast_to(utc_jd2, a.shape))
    lib().bqp_frame_tai_seconds(a.size, dptr(a), None if b is None else dptr(b), dptr(out))
    return out


def _eop_args(eop, first_mjd):
    if eop is None or len(eop) == 0:
        return None, 0, 0
    e = f64(eop).reshape(-1, 5)
    return e, int(first_mjd), e.shape[0]


def frame_matrix(epoch, policy=0, offset=0.0, eop=None, first_mjd=0):
    """R (GCRS->ITRS) of the exact chain at a UTC calendar instant
    (y, m, d, hh, mm, ss) plus `offset` s; policy 0 zero EOP, 1 the records."""
    e, f, n = _eop_args(eop, first_mjd)
    r = np.zeros(9)
    rc = lib().bqp_frame_matrix(*[int(v) for v in epoch[:5]], float(epoch[5]), int(policy), float(offset),
                                None if e is None else dptr(e), f, n, dptr(r))
    if rc != 0:
        raise ValueError(f"frame chain failed ({rc})")
    return r.reshape(3, 3)


def frame_derivatives(epoch, policy=0, h=0.25, eop=None, first_mjd=0):
    """R, Rdot, Rddot of the exact chain from its five-point stencil."""
    e, f, n = _eop_args(eop, first_mjd)
    r, rd, rdd = np.zeros(9), np.zeros(9), np.zeros(9)
    rc = lib().bqp_frame_derivatives(*[int(v) for v in epoch[:5]], float(epoch[5]), int(policy), float(h),
                                     None if e is None else dptr(e), f, n, dptr(r), dptr(rd), dptr(rdd))
    if rc != 0:
        raise ValueError(f"frame chain failed ({rc})")
    return r.reshape(3, 3), rd.reshape(3, 3), rdd.reshape(3, 3)


def frame_transform_state(epoch, r, v, a, policy=0, h=0.25, eop=None, first_mjd=0):
    """A GCRS position, velocity and acceleration in ITRS at a UTC calendar
    instant (y, m, d, hh, mm, ss), through the exact chain's stencil."""
    e, f, n = _eop_args(eop, first_mjd)
    rv, vv, av = f64(r).reshape(3), f64(v).reshape(3), f64(a).reshape(3)
    ro, vo, ao = np.zeros(3), np.zeros(3), np.zeros(3)
    rc = lib().bqp_frame_transform_state(*[int(x) for x in epoch[:5]], float(epoch[5]), int(policy), float(h),
                                         None if e is None else dptr(e), f, n, dptr(rv), dptr(vv), dptr(av),
                                         dptr(ro), dptr(vo), dptr(ao))
    if rc != 0:
        raise ValueError(f"frame chain failed ({rc})")
    return ro, vo, ao


def eop_from_finals(finals):
    """(records [n][5], first_mjd) from IERS finals2000A text (str, bytes or
    a path): the contiguous run of complete days, in the units of the sealed
    table (x_p, y_p arcsec, UT1-UTC s, dX, dY mas).  Pass it as eop=."""
    data = _text_bytes(finals)
    first = C.c_int32(0)
    n = lib().bqp_frame_eop_from_finals(data, len(data), 0, C.byref(first), None)
    if n < 0:
        raise ValueError("finals text rejected (a day given twice)")
    rec = np.zeros((max(n, 0), 5))
    if n > 0:
        lib().bqp_frame_eop_from_finals(data, len(data), n, C.byref(first), dptr(rec))
    return rec, int(first.value)


class FrameAuthority:
    """The 1800 s segment authority on the host (no GPU)."""

    def __init__(self, eop=None, first_mjd=41684):
        e, f, n = _eop_args(eop, first_mjd)
        self._keep = e
        self._h = lib().bqp_frame_authority_new(None if e is None else dptr(e), f, n)
        if not self._h:
            raise ValueError("bad EOP records")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().bqp_frame_authority_free(h)
            self._h = None

    def intervals(self):
        o = np.zeros(98)
        check(lib().bqp_frame_authority_intervals(self._h, dptr(o)))
        n = int(o[0])
        return {"start": o[1:1 + n].copy(), "delta_at": o[49:49 + n].copy(), "span_end": o[97],
                "raw": o}

    def rotation(self, tai):
        t = f64(np.atleast_1d(tai))
        r = np.empty((t.size, 9))
        w = np.empty((t.size, 3))
        lib().bqp_frame_authority_rotation(self._h, t.size, dptr(t), dptr(r), dptr(w))
        return r.reshape(-1, 3, 3), w

    def segments(self, lo, hi, cap=1 << 16):
        keys = np.zeros(cap, dtype=np.int64)
        segs = np.zeros((cap, 60))
        m = lib().bqp_frame_authority_segments(self._h, float(lo), float(hi), cap, lptr(keys), dptr(segs))
        if m < 0:
            raise ValueError("more segments than cap")
        return keys[:m].copy(), segs[:m].copy()
