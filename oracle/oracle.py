"""ctypes wrapper around the CPU oracle (oracle/prop_oracle.cpp).

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and bench.py's
CPU-baseline leg use this module as the checker.  The product package
(``bqp_b200``) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libprop_oracle.so"

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_long)

METHOD = {"dopri5_solver": 0, "dop853": 1, "dopri5": 2, "vern7": 3, "vern9": 4}  # same names as bqp_b200._native.METHODS


def build(force: bool = False) -> Path:
    srcs = [HERE / "prop_oracle.cpp", HERE / "ref_tableaus.h"]
    if force or not LIB_PATH.exists() or any(LIB_PATH.stat().st_mtime < s.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB_PATH))
        L.orc_force_new.restype = C.c_void_p
        L.orc_force_new.argtypes = [C.c_char_p, _dp]
        L.orc_force_free.argtypes = [C.c_void_p]
        L.orc_force_set_atm_model.argtypes = [C.c_void_p, C.c_int]
        L.orc_field_dense.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_gravity_itrs.argtypes = [C.c_void_p, C.c_long, _dp, _dp]
        L.orc_utc_jd_at.restype = C.c_double
        L.orc_utc_jd_at.argtypes = [C.c_double, C.c_double]
        L.orc_gmst.restype = C.c_double
        L.orc_gmst.argtypes = [C.c_double]
        L.orc_eci2equinoc.argtypes = [_dp, _dp]
        L.orc_equinoc2eci.argtypes = [_dp, C.c_double, _dp]
        L.orc_sun_moon.argtypes = [C.c_double, _dp, _dp]
        L.orc_jb2008_model.restype = C.c_double
        L.orc_jb2008_model.argtypes = [_dp, C.c_int]
        L.orc_jb2008.restype = C.c_double
        L.orc_jb2008.argtypes = [_dp]
        L.orc_geodetic_altitude_km.restype = C.c_double
        L.orc_geodetic_altitude_km.argtypes = [_dp, C.c_double]
        L.orc_rhs.argtypes = [C.c_void_p, _dp, C.c_double, C.c_double, C.c_double, C.c_double,
                              C.c_double, _dp, _dp]
        L.orc_propagate_final_batch.argtypes = [C.c_void_p, _dp, C.c_long, _dp, _dp, _dp, _dp,
                                                _dp, _ip, _lp, _lp, C.c_int]
        L.orc_propagate_sampled_batch.argtypes = [C.c_void_p, _dp, C.c_long, _dp, _dp, _dp, _dp, _dp, C.c_int,
                                                  _dp, _ip, _lp, _lp, _ip, C.c_int]
        L.orc_propagate_sampled.restype = C.c_int
        L.orc_propagate_sampled.argtypes = [C.c_void_p, _dp, _dp, C.c_double, C.c_double,
                                            C.c_double, C.c_double, _dp, C.c_int, _dp, _lp, _ip]
        L.orc_integrate_segment.restype = C.c_int
        L.orc_integrate_segment.argtypes = [C.c_void_p, _dp, _dp, C.c_double, C.c_double,
                                            C.c_double, C.c_double, C.c_double, _dp, _lp]
        L.orc_force_set_drivers.restype = C.c_int
        L.orc_force_set_drivers.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_char_p, C.c_int]
        L.orc_jb_lookup.restype = C.c_int
        L.orc_jb_lookup.argtypes = [C.c_void_p, C.c_long, _dp, _dp, _ip]
        L.orc_force_set_ephemeris.restype = C.c_int
        L.orc_force_set_ephemeris.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_long, C.c_char_p, C.c_int]
        L.orc_body_positions.restype = None
        L.orc_body_positions.argtypes = [C.c_void_p, C.c_int, C.c_long, _dp, _dp]
        L.orc_shadow_cylinder.restype = C.c_int
        L.orc_shadow_cylinder.argtypes = [_dp, _dp, C.c_double, _dp]
        L.orc_srp_accel.restype = None
        L.orc_srp_accel.argtypes = [_dp, _dp, C.c_double, C.c_double, C.c_double, C.c_int, _dp]
        L.orc_eclipse_envelope_ok.restype = C.c_int
        L.orc_eclipse_envelope_ok.argtypes = [_dp, _dp]
        L.orc_no_crossing_certified.restype = C.c_int
        L.orc_no_crossing_certified.argtypes = [C.c_double, C.c_double, C.c_double]
        L.orc_first_crossing_in_step.restype = C.c_int
        L.orc_first_crossing_in_step.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.c_long,
                                                 _STATE_FN, _BOUND_FN, _dp, _lp]
        L.orc_drivers_counts.restype = C.c_int
        L.orc_drivers_counts.argtypes = [C.c_void_p, _lp]
        L.orc_force_set_srp.restype = None
        L.orc_force_set_srp.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
        L.orc_sun_rate_bound.restype = C.c_double
        L.orc_sun_rate_bound.argtypes = [C.c_void_p]
        L.orc_propagate_srp_roots.restype = C.c_int
        L.orc_propagate_srp_roots.argtypes = [C.c_void_p, _dp, _dp, C.c_double, C.c_double, C.c_double, C.c_double,
                                              _dp, _dp, C.c_int, _ip, _lp]
        L.orc_ecl_decisive_margin.restype = C.c_int
        L.orc_ecl_decisive_margin.argtypes = [C.c_double, _dp]
        L.orc_ecl_replay_unc.restype = C.c_int
        L.orc_ecl_replay_unc.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, _dp]
        L.orc_ecl_deepest.restype = C.c_int
        L.orc_ecl_deepest.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_double, _dp]
        L.orc_propagate_srp_batch.restype = None
        L.orc_propagate_srp_batch.argtypes = [C.c_void_p, _dp, C.c_long, _dp, _dp, _dp, _dp, _dp, C.c_int,
                                              _dp, _dp, _ip, _lp, _lp, _ip, C.c_int]
        L.orc_force_set_frame.restype = None
        L.orc_force_set_frame.argtypes = [C.c_void_p, C.c_long, C.POINTER(C.c_int64), _dp, _dp]
        L.orc_frame_rotation.restype = C.c_int
        L.orc_frame_rotation.argtypes = [C.c_void_p, C.c_long, _dp, _dp, _dp]
        L.orc_frame_tai_origin.restype = C.c_double
        L.orc_frame_tai_origin.argtypes = [C.c_double]
        _lib = L
    return _lib


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class Force:
    """A force model: gravity field (normalised ``deg ord C S`` text) plus switches."""

    def __init__(self, coeff_text: str, order: int, drag=False, sun=False, moon=False,
                 earth_radius=6378.137, omega=7.292115e-5, mu_sun=1.32712440018e11,
                 mu_moon=4902.800066, drivers=(150.0,) * 8 + (0.0,), atm_model=4):
        cfg = f64([order, int(drag), int(sun), int(moon), earth_radius, omega, mu_sun, mu_moon,
                   *drivers])
        self.order = order
        self.h = lib().orc_force_new(coeff_text.encode(), _d(cfg))
        if not self.h:
            raise ValueError("oracle: coefficient text rejected")
        if lib().orc_force_set_atm_model(self.h, int(atm_model)) != 0:
            raise ValueError(f"oracle: atm_model {atm_model} is not 4, 5, 6 or 7")

    def set_frame(self, keys=None, segs=None, intervals=None):
        """The Earth-fixed frame: IAU 2006/2000A segments (keys [n] int64,
        segs [n][60], intervals [98] as the library exports them), or GMST
        when keys is None.  The segments are an input: this restates their
        lookup and evaluation only."""
        if keys is None:
            lib().orc_force_set_frame(self.h, -1, None, None, None)
            return
        k = np.ascontiguousarray(keys, dtype=np.int64)
        sg = f64(segs).reshape(-1, 60)
        iv = f64(intervals).reshape(98)
        lib().orc_force_set_frame(self.h, k.size, k.ctypes.data_as(C.POINTER(C.c_int64)), _d(sg), _d(iv))

    def frame_rotation(self, tai):
        t = f64(np.atleast_1d(tai))
        r = np.zeros((t.size, 9))
        w = np.zeros((t.size, 3))
        lib().orc_frame_rotation(self.h, t.size, _d(t), _d(r), _d(w))
        return r.reshape(-1, 3, 3), w

    def set_srp(self, on=True, cr=1.3, p_sun=4.56e-6):
        """Solar radiation pressure with the binary-eclipse coordinator (rows
        whose A/m, cr and p_sun are all > 0)."""
        lib().orc_force_set_srp(self.h, int(bool(on)), float(cr), float(p_sun))

    def sun_rate_bound(self) -> float:
        """Upper bound of the Sun direction's angular rate, rad/day."""
        return float(lib().orc_sun_rate_bound(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_force_free(self.h)
            self.h = None

    def set_drivers(self, solfsmy: str | None, dtcfile: str | None):
        """Look the JB2008 drivers up per evaluation in these SOLFSMY / DTCFILE
        texts (None, None: back to the fixed drivers); ValueError on a
        rejected file."""
        err = C.create_string_buffer(256)
        rc = lib().orc_force_set_drivers(self.h, None if solfsmy is None else solfsmy.encode(),
                                         None if dtcfile is None else dtcfile.encode(), err, 256)
        if rc != 0:
            raise ValueError(f"oracle: space-weather file rejected: {err.value.decode()}")

    def jb_lookup(self, utc_jd):
        """(drivers [n, 9] with NaN rows where the lookup fails, ok [n] bool)."""
        jd = f64(np.atleast_1d(utc_jd))
        out = np.zeros((jd.size, 9))
        ok = np.zeros(jd.size, dtype=np.int32)
        if lib().orc_jb_lookup(self.h, jd.size, _d(jd), _d(out), ok.ctypes.data_as(_ip)) != 0:
            raise ValueError("oracle: no space-weather tables set")
        return out, ok.astype(bool)

    def set_ephemeris(self, body: str, data: bytes | None):
        """Sun or Moon positions from a precomputed catalogue ("DUST" format;
        None: back to the analytic series); ValueError on a rejected file."""
        err = C.create_string_buffer(256)
        b = {"sun": 0, "moon": 1}[body]
        if lib().orc_force_set_ephemeris(self.h, b, data, 0 if data is None else len(data), err, 256) != 0:
            raise ValueError(f"oracle: ephemeris catalogue rejected: {err.value.decode()}")

    def body_positions(self, body: str, utc_jd):
        jd = f64(np.atleast_1d(utc_jd))
        out = np.zeros((jd.size, 3))
        lib().orc_body_positions(self.h, {"sun": 0, "moon": 1}[body], jd.size, _d(jd), _d(out))
        return out

    def driver_counts(self):
        c = np.zeros(2, dtype=np.int64)
        if lib().orc_drivers_counts(self.h, c.ctypes.data_as(_lp)) != 0:
            raise ValueError("oracle: no space-weather tables set")
        return int(c[0]), int(c[1])

    def dense(self):
        st = self.order + 2
        c = np.zeros(st * st)
        s = np.zeros(st * st)
        lib().orc_field_dense(self.h, _d(c), _d(s))
        return c.reshape(st, st), s.reshape(st, st)

    def gravity_itrs(self, pos_km: np.ndarray) -> np.ndarray:
        p = f64(pos_km).reshape(-1, 3)
        out = np.zeros_like(p)
        lib().orc_gravity_itrs(self.h, p.shape[0], _d(p), _d(out))
        return out

    def rhs(self, eq, t0, jd0, am, cd, t, delta):
        eq = f64(eq)
        delta = f64(delta)
        out = np.zeros(6)
        lib().orc_rhs(self.h, _d(eq), t0, jd0, am, cd, t, _d(delta), _d(out))
        return out


def ctrl(method="dop853", eps=1e-8, rtol=None, atol=None, dt_max=300.0, max_steps=500000):
    scaled = rtol is not None
    return f64([METHOD[method], 1 if scaled else 0, eps, rtol or 0.0, atol or 0.0, dt_max,
                max_steps])


def propagate_final_batch(force: Force, ctl, eq0, epoch_jd, tf, ballistic, threads=0):
    eq0 = f64(eq0).reshape(-1, 6)
    n = eq0.shape[0]
    epoch_jd = f64(np.broadcast_to(epoch_jd, (n,)))
    tf = f64(np.broadcast_to(tf, (n,)))
    ballistic = f64(np.broadcast_to(ballistic, (n, 2)))
    out = np.zeros((n, 6))
    status = np.zeros(n, dtype=np.int32)
    steps = np.zeros(n, dtype=np.int64)
    evals = np.zeros(n, dtype=np.int64)
    lib().orc_propagate_final_batch(force.h, _d(f64(ctl)), n, _d(eq0), _d(epoch_jd), _d(tf),
                                    _d(ballistic), _d(out), status.ctypes.data_as(_ip),
                                    steps.ctypes.data_as(_lp), evals.ctypes.data_as(_lp),
                                    int(threads))
    return out, status, steps, evals


def propagate_sampled(force: Force, ctl, eq0, epoch_jd, tf, am, cd, t_eval):
    t_eval = f64(t_eval)
    out = np.full((t_eval.size, 6), np.nan)
    se = np.zeros(2, dtype=np.int64)
    nw = C.c_int(0)
    st = lib().orc_propagate_sampled(force.h, _d(f64(ctl)), _d(f64(eq0)), epoch_jd, tf, am, cd,
                                     _d(t_eval), t_eval.size, _d(out), se.ctypes.data_as(_lp),
                                     C.byref(nw))
    return out, st, int(se[0]), int(se[1]), nw.value


def propagate_sampled_batch(force: Force, ctl, eq0, epoch_jd, tf, ballistic, t_eval, threads=0):
    """Sampled path of n rows on one grid, all host threads: (delta [n][n_t][6]
    against each row's initial baseline, status[n], steps[n], evals[n],
    samples written[n])."""
    eq0 = f64(eq0).reshape(-1, 6)
    n = eq0.shape[0]
    epoch_jd = f64(np.broadcast_to(epoch_jd, (n,)))
    tf = f64(np.broadcast_to(tf, (n,)))
    ballistic = f64(np.broadcast_to(ballistic, (n, 2)))
    t_eval = f64(t_eval)
    out = np.empty((n, t_eval.size, 6))
    status = np.zeros(n, dtype=np.int32)
    steps = np.zeros(n, dtype=np.int64)
    evals = np.zeros(n, dtype=np.int64)
    nw = np.zeros(n, dtype=np.int32)
    lib().orc_propagate_sampled_batch(force.h, _d(f64(ctl)), n, _d(eq0), _d(epoch_jd), _d(tf), _d(ballistic),
                                      _d(t_eval), t_eval.size, _d(out), status.ctypes.data_as(_ip),
                                      steps.ctypes.data_as(_lp), evals.ctypes.data_as(_lp),
                                      nw.ctypes.data_as(_ip), int(threads))
    return out, status, steps, evals, nw


# eclipse coordinator status words (EclipseError)
ECLIPSE_STATUS = {11: "envelope", 12: "chatter", 13: "bracket", 14: "non_progress", 15: "geometry",
                  16: "split_limit"}


def propagate_srp_batch(force: Force, ctl, eq0, epoch_jd, tf, ballistic, t_eval=None, threads=0):
    """Rows through the binary-eclipse coordinator (force.set_srp first):
    (final delta [n][6] against each row's initial baseline, samples
    [n][n_t][6] or None, status[n], steps[n], evals[n], samples written[n])."""
    eq0 = f64(eq0).reshape(-1, 6)
    n = eq0.shape[0]
    epoch_jd = f64(np.broadcast_to(epoch_jd, (n,)))
    tf = f64(np.broadcast_to(tf, (n,)))
    ballistic = f64(np.broadcast_to(ballistic, (n, 2)))
    te = f64(t_eval) if t_eval is not None else np.zeros(0)
    out = np.zeros((n, 6))
    smp = np.empty((n, te.size, 6)) if t_eval is not None else None
    status = np.zeros(n, dtype=np.int32)
    steps = np.zeros(n, dtype=np.int64)
    evals = np.zeros(n, dtype=np.int64)
    nw = np.zeros(n, dtype=np.int32)
    lib().orc_propagate_srp_batch(force.h, _d(f64(ctl)), n, _d(eq0), _d(epoch_jd), _d(tf), _d(ballistic),
                                  _d(te) if te.size else None, int(te.size), _d(out),
                                  _d(smp) if smp is not None else None, status.ctypes.data_as(_ip),
                                  steps.ctypes.data_as(_lp), evals.ctypes.data_as(_lp), nw.ctypes.data_as(_ip),
                                  int(threads))
    return out, smp, status, steps, evals, nw


def propagate_srp_roots(force: Force, ctl, eq0, epoch_jd, tf, am, cd, max_roots=4096):
    """One row through the coordinator: (final delta, committed root instants,
    status, steps, evals)."""
    d = np.zeros(6)
    roots = np.zeros(max_roots)
    nr = C.c_int(0)
    se = np.zeros(2, dtype=np.int64)
    st = lib().orc_propagate_srp_roots(force.h, _d(f64(ctl)), _d(f64(eq0)), float(epoch_jd), float(tf), float(am),
                                       float(cd), _d(d), _d(roots), max_roots, C.byref(nr), se.ctypes.data_as(_lp))
    return d, roots[:min(nr.value, max_roots)].copy(), st, int(se[0]), int(se[1])


def ecl_decisive_margin(err):
    out = C.c_double(0.0)
    st = lib().orc_ecl_decisive_margin(float(err), C.byref(out))
    return (out.value if st == 0 else None), st


def ecl_replay_uncertainty(force: Force, epoch_jd, t0, t1):
    out = C.c_double(0.0)
    st = lib().orc_ecl_replay_unc(force.h, float(epoch_jd), float(t0), float(t1), C.byref(out))
    return (out.value if st == 0 else None), st


def ecl_deepest(force: Force, epoch_jd, old_t, lim, max_km):
    out = C.c_double(0.0)
    st = lib().orc_ecl_deepest(force.h, float(epoch_jd), float(old_t), float(lim), float(max_km), C.byref(out))
    return (out.value if st == 0 else None), st


def integrate_segment(force: Force, ctl, eq, jd0, am, cd, t0, tf):
    y = np.zeros(6)
    se = np.zeros(2, dtype=np.int64)
    st = lib().orc_integrate_segment(force.h, _d(f64(ctl)), _d(f64(eq)), jd0, am, cd, t0, tf,
                                     _d(y), se.ctypes.data_as(_lp))
    return y, st, int(se[0]), int(se[1])


def eci2equinoc(eci):
    out = np.zeros(6)
    rc = lib().orc_eci2equinoc(_d(f64(eci)), _d(out))
    return out, rc


def equinoc2eci(eq, tof):
    out = np.zeros(6)
    rc = lib().orc_equinoc2eci(_d(f64(eq)), tof, _d(out))
    return out, rc


def utc_jd_at(jd0, t):
    """UTC Julian day t elapsed (TAI) seconds after the UTC epoch jd0."""
    return lib().orc_utc_jd_at(float(jd0), float(t))


def gmst(jd):
    return lib().orc_gmst(jd)


def sun_moon(jd):
    s = np.zeros(3)
    m = np.zeros(3)
    lib().orc_sun_moon(jd, _d(s), _d(m))
    return s, m


def jb2008_model(inputs14, model: int) -> float:
    """JB2008 density of atm_model 4 (exact), 5, 6 or 7; negative: an error code."""
    return lib().orc_jb2008_model(_d(f64(inputs14)), int(model))


def jb2008(inputs14) -> float:
    return lib().orc_jb2008(_d(f64(inputs14)))


def geodetic_altitude_km(pos_km, a=6378.137) -> float:
    return lib().orc_geodetic_altitude_km(_d(f64(pos_km)), a)


# ---------------------------------------------------- SRP and the shadow cylinder
def shadow_cylinder(sat, sun, earth_radius=6378.137):
    """("shadow" | "lit", margin km) of the Earth's shadow cylinder, or None for
    invalid geometry."""
    out = np.zeros(2)
    if lib().orc_shadow_cylinder(_d(f64(sat)), _d(f64(sun)), float(earth_radius), _d(out)) != 0:
        return None
    return ("shadow" if out[0] else "lit"), float(out[1])


def srp_accel(sat, sun, cr=1.3, am=0.01, shadow=False, p_sun=4.56e-6):
    out = np.zeros(3)
    lib().orc_srp_accel(_d(f64(sat)), _d(f64(sun)), float(p_sun), float(cr), float(am), int(bool(shadow)), _d(out))
    return out


def eclipse_envelope_ok(pos, vel) -> bool:
    return bool(lib().orc_eclipse_envelope_ok(_d(f64(pos)), _d(f64(vel))))


_STATE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_double, _dp, _dp, _dp)
_BOUND_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, _dp, _dp, _dp)
SCAN_ERRORS = {1: "geometry", 2: "bracket", 3: "non_progress", 4: "split_limit"}


def first_crossing_in_step(t_old, t_new, state, bound, max_splits=1_000_000, earth_radius=6378.137,
                           max_sep=1.0e-6):
    """The oracle's shadow-crossing scan.  state(t) -> (pos, vel, sun) or None
    for failure; bound((t, pos, vel), (t, pos, vel)) -> km or None.  Returns
    (error name or None, result dict)."""

    def c_state(_, t, pos, vel, sun):
        got = state(t)
        if got is None:
            return 1
        for dst, src in zip((pos, vel, sun), got):
            for i in range(3):
                dst[i] = float(src[i])
        return 0

    def c_bound(_, a, b, out):
        got = bound((a[0], tuple(a[1:4]), tuple(a[4:7])), (b[0], tuple(b[1:4]), tuple(b[4:7])))
        if got is None:
            return 1
        out[0] = float(got)
        return 0

    sf, bf = _STATE_FN(c_state), _BOUND_FN(c_bound)
    out = np.zeros(6)
    collapsed = np.zeros(1, dtype=np.int64)
    e = lib().orc_first_crossing_in_step(float(t_old), float(t_new), float(earth_radius), float(max_sep),
                                         int(max_splits), sf, bf, _d(out), collapsed.ctypes.data_as(_lp))
    res = {"found": bool(out[0]), "t_old": out[1], "t_new": out[2],
           "old_side": "shadow" if out[3] else "lit", "new_side": "shadow" if out[4] else "lit",
           "bound": out[5], "collapsed_pairs": int(collapsed[0])}
    return SCAN_ERRORS.get(e), res


def no_crossing_certified(m_old, m_new, bound) -> bool:
    return bool(lib().orc_no_crossing_certified(float(m_old), float(m_new), float(bound)))


def frame_tai_origin(jd0: float) -> float:
    """Continuous TAI seconds of t = 0 for a one-part UTC epoch (NaN before 1972)."""
    return float(lib().orc_frame_tai_origin(float(jd0)))
