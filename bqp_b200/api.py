"""The ``dust_transfer`` propagator surface, on the B200 propagator.

Same names, keyword arguments, defaults, dict keys and exceptions as the
reference binding (dust_transfer/src/lib.rs:200-438 and
python/dust_transfer/__init__.py):

    propagate(state_eci, epoch_jd, tof_s, times_s=None, *, gravity_order=5, drag=True,
              srp=True, sun=True, moon=True, atm_model=7, am_ratio=0.01, cd=2.2, cr=1.3,
              tol=1e-8, dt_max_s=300.0, method="vern7") -> dict
    propagate_final(...) -> np.ndarray (6,)
    kep_to_eci(kep) / eci_to_kep(eci)

plus batch entry points (the reference's Rust batch/session APIs, which the
Python binding does not expose): ``propagate_batch_final`` and
``propagate_batch_sampled``.

Options this build does not implement raise ``ValueError`` naming the option
(the tsit5/rkv98 tableaus, SRP with the dopri5 compatibility stepper or
rtol/atol control); they are never silently replaced.  ``gravity_field`` (extra keyword) takes a normalised
``deg ord C S`` text or a path, which lifts the embedded field's degree-15 cap.

Extra keywords for the inputs the reference reads from its own tree:
``space_weather`` (SET SOLFSMY / DTCFILE), ``ephemeris`` (Sun / Moon "DUST"
catalogues) and ``eop`` (the sealed EOP table or IERS finals2000A text) for
the Earth-fixed frame, which is the reference's IAU 2006/2000A chain
(``frame="iau2006"``, the default; zero EOP without ``eop``) or the GMST
z-rotation (``frame="gmst"``).
"""
from __future__ import annotations

import hashlib
import time
import warnings
from collections import OrderedDict
from pathlib import Path

import numpy as np

from . import _native as N

MU_EARTH_KM3_S2 = 398600.4415
SEC_PER_DAY = 86400.0
MAX_GRAVITY_ORDER = 15  # embedded DIR-R6 field (lib.rs:53)
DATA = Path(__file__).resolve().parent / "data"
_DEFAULT_FIELD = DATA / "dir_r6_d15.txt"

_UNBUILT_METHODS = ("tsit5", "rkv98")
_METHODS = {"dop853": N.METHODS["dop853"], "dopri5": N.METHODS["dopri5"],
            "dopri5_solver": N.METHODS["dopri5_solver"], "vern7": N.METHODS["vern7"],
            "vern9": N.METHODS["vern9"]}


def _six(value, what):
    try:
        v = np.asarray(value, dtype=np.float64).reshape(-1)
    except (TypeError, ValueError):
        raise ValueError(f"{what} must be a sequence of 6 floats") from None
    if v.size != 6:
        raise ValueError(f"{what} must have exactly 6 elements")
    if not np.all(np.isfinite(v)):
        raise ValueError(f"{what} contains a non-finite value")
    return v


def _field_text(gravity_field) -> tuple[str, bool]:
    if gravity_field is None:
        return _DEFAULT_FIELD.read_text(), True
    if isinstance(gravity_field, Path) or (isinstance(gravity_field, str) and "\n" not in gravity_field
                                           and Path(gravity_field).exists()):
        return Path(gravity_field).read_text(), False
    if isinstance(gravity_field, str):
        return gravity_field, False
    raise ValueError("gravity_field must be coefficient text or a path")


def force_config(gravity_order=5, drag=True, srp=True, sun=True, moon=True, atm_model=7, am_ratio=0.01,
                 cd=2.2, cr=1.3, tol=1e-8, dt_max_s=300.0, method="vern7", embedded=True,
                 rtol=None, atol=None, jb_drivers=None, ground_check=False) -> N.ForceConfig:
    """The reference's force_config() (lib.rs:128-190) onto bqp_force_config."""
    limit = MAX_GRAVITY_ORDER if embedded else 128
    if not (isinstance(gravity_order, (int, np.integer)) and 1 <= gravity_order <= limit):
        raise ValueError(f"gravity_order must be in 1..={limit}, got {gravity_order}")
    if not (np.isfinite(am_ratio) and am_ratio > 0 and np.isfinite(cd) and cd > 0 and np.isfinite(cr) and cr >= 0):
        raise ValueError("am_ratio and cd must be finite and > 0, cr finite and >= 0")
    if not (np.isfinite(tol) and tol > 0 and np.isfinite(dt_max_s) and dt_max_s > 0):
        raise ValueError("tol and dt_max_s must be finite and > 0")
    if drag and atm_model not in (1, 3, 4, 5, 6, 7, 8):
        raise ValueError(f"unknown atm_model {atm_model}; use 4 (exact JB2008), 7 (fitted JB2008), "
                         "8 (campaign persistence scenario), 1 (exponential)")
    if drag and atm_model not in (4, 5, 6, 7):
        raise ValueError(f"atm_model {atm_model} is not built here; use 4 (exact JB2008) or 5, 6, 7 (the "
                         "coarse JB2008 quadrature profiles, 7 the fitted kernel)")
    name = str(method).lower()
    if name in _UNBUILT_METHODS:
        raise ValueError(f"integrator method {name!r} is not built here; use 'vern7', 'vern9', 'dop853' or 'dopri5'")
    if name not in _METHODS:
        raise ValueError(f"unknown integrator method {name!r}; use one of vern7, vern9, dop853, tsit5, rkv98, "
                         "dopri5")
    if srp and name == "dopri5":
        raise ValueError("srp=True runs the binary-eclipse coordinator with vern7, vern9 or dop853 here, not the "
                         "dopri5 compatibility stepper; pass srp=False or another method")
    if srp and rtol is not None:
        raise ValueError("srp=True runs with the absolute tolerance tol here, not rtol/atol")
    cfg = N.default_config()
    cfg.order = int(gravity_order)
    flags = 0
    if drag:
        flags |= N.FORCE_DRAG
    if sun:
        flags |= N.FORCE_SUN
    if moon:
        flags |= N.FORCE_MOON
    if srp:
        flags |= N.FORCE_SRP
    cfg.force_flags = flags
    cfg.cr = float(cr)
    cfg.atm_model = int(atm_model) if drag else 0
    cfg.method = _METHODS[name]
    cfg.am_ratio = float(am_ratio)
    cfg.cd = float(cd)
    cfg.dt_max = float(dt_max_s)
    if rtol is not None:
        cfg.error_control = 1
        cfg.rtol = float(rtol)
        cfg.atol = float(atol if atol is not None else 0.0)
    else:
        cfg.error_control = 0
        cfg.eps = float(tol)
    if jb_drivers is not None:
        for i, v in enumerate(jb_drivers):
            cfg.jb_drivers[i] = float(v)
    cfg.ground_check = 1 if ground_check else 0
    return cfg


# ------------------------------------------------------------------ contexts
_CTX: "OrderedDict[tuple, N.Context]" = OrderedDict()
_CTX_MAX = 8


def _cfg_key(cfg: N.ForceConfig):
    return tuple(getattr(cfg, f) if f != "jb_drivers" else tuple(cfg.jb_drivers) for f, _ in cfg._fields_)


def _space_weather(space_weather):
    """(SOLFSMY bytes, DTCFILE bytes, span) of space_weather = (solfsmy,
    dtcfile) or (solfsmy, dtcfile, (jd_lo, jd_hi)); each file as text, bytes
    or a path."""
    if space_weather is None:
        return None
    if not isinstance(space_weather, (tuple, list)) or len(space_weather) not in (2, 3):
        raise ValueError("space_weather must be (solfsmy, dtcfile) or (solfsmy, dtcfile, (jd_lo, jd_hi))")
    span = tuple(float(x) for x in space_weather[2]) if len(space_weather) == 3 else (0.0, 0.0)
    return N._text_bytes(space_weather[0]), N._text_bytes(space_weather[1]), span


def _ephemeris(ephemeris):
    """{"sun": bytes, "moon": bytes} of ephemeris = (sun, moon) (either may be
    None) or a dict with those keys; each catalogue as bytes or a path."""
    if ephemeris is None:
        return {}
    if isinstance(ephemeris, dict):
        items = ephemeris.items()
    elif isinstance(ephemeris, (tuple, list)) and len(ephemeris) == 2:
        items = zip(("sun", "moon"), ephemeris)
    else:
        raise ValueError("ephemeris must be (sun, moon) or {'sun': ..., 'moon': ...}")
    out = {}
    for body, cat in items:
        if body not in N.BODIES:
            raise ValueError(f"unknown ephemeris body {body!r}")
        if cat is not None:
            out[body] = N._file_bytes(cat)
    return out


_ZERO_EOP_WARNED = False  # the zero-EOP notice is given once per process


def _frame(frame, eop):
    """(frame name, EOP records [n][5] or None, first MJD) of frame= / eop=.
    eop: None (zero EOP), the bytes or path of a sealed EOP table (five
    little-endian binary64 per UTC day from MJD 41684, the reference's
    frame_time/eop_table.bin) or of IERS finals2000A text (told apart by
    being ASCII lines), or (records [n][5], first_mjd)."""
    global _ZERO_EOP_WARNED
    if frame not in N.FRAMES:
        raise ValueError(f"frame must be one of {sorted(N.FRAMES)}, got {frame!r}")
    if eop is None:
        if frame == "iau2006" and not _ZERO_EOP_WARNED:
            _ZERO_EOP_WARNED = True
            warnings.warn("the IAU 2006/2000A frame runs with zero EOP (UT1-UTC = polar motion = 0): pass "
                          "eop= the reference's eop_table.bin or IERS finals2000A text for its Earth orientation",
                          UserWarning, stacklevel=4)
        return frame, None, 41684
    if frame != "iau2006":
        raise ValueError("eop is for frame='iau2006'")
    if isinstance(eop, tuple) and len(eop) == 2:
        rec = np.asarray(eop[0], dtype=np.float64).reshape(-1, 5)
        return frame, rec, int(eop[1])
    data = eop.encode() if isinstance(eop, str) and "\n" in eop else N._file_bytes(eop)
    head = data[:4096]
    if b"\n" in head and head.isascii():
        rec, first = N.eop_from_finals(data)
        if rec.shape[0] == 0:
            raise ValueError("no complete finals2000A row in the EOP text")
        return frame, rec, first
    if len(data) % 40:
        raise ValueError("a sealed EOP table holds 40-byte records")
    return frame, np.frombuffer(data, dtype="<f8").reshape(-1, 5).astype(np.float64), 41684


def context(text: str, cfg: N.ForceConfig, space_weather=None, ephemeris=None, frame="iau2006",
            eop=None) -> N.Context:
    """A cached native context for (field text, configuration, space-weather
    files, ephemeris catalogues).  With space_weather the JB2008 drivers come
    from the SET SOLFSMY / DTCFILE tables at each evaluation's UTC instant (the
    reference's compiled driver catalogue, jb_rs/src/drivers.rs) instead of
    the fixed configured drivers; with ephemeris the Sun and / or Moon come
    from precomputed "DUST" catalogues (the reference's precomputed_ephem.rs)
    instead of the analytic series.  Gravity and drag take the Earth-fixed
    frame from the IAU 2006/2000A chain (frame="iau2006", the reference's
    frame authority, satpy_core/src/frame_time/authority.rs) with the EOP
    records of eop (zero EOP when None), or from the GMST rotation
    (frame="gmst")."""
    sw = _space_weather(space_weather)
    eph = _ephemeris(ephemeris)
    fr = _frame(frame, eop)
    sw_key = None if sw is None else (hashlib.sha256(sw[0]).hexdigest(), hashlib.sha256(sw[1]).hexdigest(), sw[2])
    eph_key = tuple(sorted((b, hashlib.sha256(d).hexdigest()) for b, d in eph.items()))
    fr_key = (fr[0], None if fr[1] is None else hashlib.sha256(fr[1].tobytes()).hexdigest(), fr[2])
    key = (hashlib.sha256(text.encode()).hexdigest(), _cfg_key(cfg), sw_key, eph_key, fr_key)
    ctx = _CTX.get(key)
    if ctx is None:
        ctx = N.Context(text, cfg)
        if sw is not None:
            ctx.set_jb_drivers(sw[0], sw[1], sw[2])
        for body, data in eph.items():
            ctx.set_ephemeris(body, data)
        if fr[0] != "gmst":
            ctx.set_frame(fr[0], fr[1], fr[2])
        _CTX[key] = ctx
        while len(_CTX) > _CTX_MAX:
            _CTX.popitem(last=False)[1].close()
    else:
        _CTX.move_to_end(key)
    return ctx


def _equinoctial_of(eci, what):
    equ, ok = N.eci_to_equinoctial(eci)
    if not ok[0]:
        raise ValueError(f"{what} is not a bound, non-degenerate elliptical orbit (equinoctial conversion failed)")
    return equ[0]


def _srp_in_effect(cfg) -> bool:
    """SRP acts (rhs.rs:31-36): the flag with cr, p_sun and A/m all > 0."""
    return bool(cfg.force_flags & N.FORCE_SRP) and cfg.cr > 0 and cfg.p_sun > 0 and cfg.am_ratio > 0


# ------------------------------------------------------------------ scalar API
def propagate(state_eci, epoch_jd, tof_s, times_s=None, *, gravity_order=5, drag=True, srp=True, sun=True,
              moon=True, atm_model=7, am_ratio=0.01, cd=2.2, cr=1.3, tol=1e-8, dt_max_s=300.0, method="vern7",
              gravity_field=None, space_weather=None, ephemeris=None, frame="iau2006", eop=None):
    """Propagate one ECI state; sampled, rectified path (lib.rs:237-353).

    space_weather = (solfsmy, dtcfile[, (jd_lo, jd_hi)]): JB2008 drivers from
    SET space-weather files; ephemeris = (sun, moon): precomputed catalogues
    (see ``context``); defaults: the fixed drivers, the analytic series and,
    as in the reference (rhs.rs:3113-3174), the IAU 2006/2000A Earth-fixed
    frame -- with zero EOP unless eop passes the reference's sealed table or
    records (frame="gmst": the GMST z-rotation instead)."""
    init = _six(state_eci, "state_eci")
    if not (np.isfinite(epoch_jd) and np.isfinite(tof_s) and tof_s > 0):
        raise ValueError("epoch_jd must be finite and tof_s > 0")
    if times_s is None:
        user = np.array([float(tof_s)])
    else:
        try:
            user = np.asarray(times_s, dtype=np.float64).reshape(-1)
        except (TypeError, ValueError):
            raise ValueError("times_s must be a sequence of floats") from None
    if (user.size > 1 and np.any(np.diff(user) <= 0)) or np.any(~np.isfinite(user)) or np.any(user < 0) \
            or np.any(user > tof_s):
        raise ValueError("times_s must be strictly increasing, within [0, tof_s]")
    grid = []
    if user.size == 0 or user[0] > 0.0:
        grid.append(0.0)
    grid.extend(user.tolist())
    if user.size == 0 or user[-1] < tof_s:
        grid.append(float(tof_s))
    text, embedded = _field_text(gravity_field)
    cfg = force_config(gravity_order, drag, srp, sun, moon, atm_model, am_ratio, cd, cr, tol, dt_max_s,
                       method, embedded)
    _equinoctial_of(init, "state_eci")
    ctx = context(text, cfg, space_weather, ephemeris, frame, eop)
    t_start = time.perf_counter()
    out, st, steps, evals = ctx.propagate_sampled(init, epoch_jd, tof_s, np.array(grid))
    wall_us = int((time.perf_counter() - t_start) * 1e6)
    status = int(st[0])
    states = out[0]
    good = np.all(np.isfinite(states), axis=1)
    n_ok = len(grid) if status == N.ST_OK else int(np.argmin(good)) if not good.all() else len(grid)
    completed = status == N.ST_OK and n_ok == len(grid)
    if status == N.ST_OK:
        terminal = ""
    else:
        terminal = N.STATUS_NAMES.get(status, "incomplete")
    if _srp_in_effect(cfg) and (status in N.ECLIPSE_STATUSES or status == N.ST_GRAVITY_RADIUS):
        # an eclipse failure returns no samples (lib.rs:297-303, integrator.rs:2463-2473)
        n_ok = 0
        if status == N.ST_GRAVITY_RADIUS:
            terminal = "eclipse_gravity"
    return {
        "times_s": np.array(grid[:n_ok]),
        "states_eci": states[:n_ok].copy(),
        "completed": bool(completed),
        "terminal_event": terminal,
        "max_steps_exceeded": status == 1,
        "steps": int(steps[0]),
        "rhs_evals": int(evals[0]),
        "wall_us": wall_us,
    }


def propagate_final(state_eci, epoch_jd, tof_s, *, gravity_order=5, drag=True, srp=True, sun=True, moon=True,
                    atm_model=7, am_ratio=0.01, cd=2.2, cr=1.3, tol=1e-8, dt_max_s=300.0, method="vern7",
                    gravity_field=None, space_weather=None, ephemeris=None, frame="iau2006", eop=None):
    """Final state with the ground check enforced (lib.rs:361-438).

    Raises ValueError for a physically infeasible arc (ground impact, a radius
    below the surface) and RuntimeError for an integration failure."""
    init = _six(state_eci, "state_eci")
    if not (np.isfinite(epoch_jd) and np.isfinite(tof_s) and tof_s > 0):
        raise ValueError("epoch_jd must be finite and tof_s > 0")
    text, embedded = _field_text(gravity_field)
    cfg = force_config(gravity_order, drag, srp, sun, moon, atm_model, am_ratio, cd, cr, tol, dt_max_s,
                       method, embedded, ground_check=True)
    _equinoctial_of(init, "state_eci")
    ctx = context(text, cfg, space_weather, ephemeris, frame, eop)
    out, st, _, _ = ctx.propagate_final(init, epoch_jd, tof_s)
    status = int(st[0])
    if status == N.ST_GROUND:
        raise ValueError("physically infeasible arc: trajectory hits the ground")
    if status == N.ST_GRAVITY_RADIUS:
        raise ValueError("physically infeasible arc: radius fell below the Earth's surface")
    if status == N.ST_ECLIPSE_ENVELOPE:
        raise ValueError("state outside the SRP eclipse envelope (radius 6000-50000 km, speed <= 20 km/s); "
                         "pass srp=False")
    if status != N.ST_OK:
        raise RuntimeError(f"propagation failed: {N.STATUS_NAMES.get(status, status)}")
    return out[0].copy()


def kep_to_eci(kep):
    """Keplerian [a_km, e, i_deg, raan_deg, argp_deg, true_anomaly_deg] -> ECI (lib.rs:200-211)."""
    k = _six(kep, "kep")
    if k[0] <= 0.0 or not (0.0 <= k[1] < 1.0):
        raise ValueError("need a_km > 0 and 0 <= e < 1")
    return N.kep_to_eci(k)[0]


def eci_to_kep(eci):
    """ECI (km, km/s) -> Keplerian elements in degrees (lib.rs:213-221)."""
    return N.eci_to_kep(_six(eci, "eci"))[0]


# ------------------------------------------------------------------ batch API
def _batch_cfg(model: dict, embedded: bool):
    m = dict(gravity_order=5, drag=True, srp=False, sun=True, moon=True, atm_model=7, am_ratio=0.01, cd=2.2,
             cr=1.3, tol=1e-8, dt_max_s=300.0, method="dop853")
    m.update(model)
    return force_config(m["gravity_order"], m["drag"], m["srp"], m["sun"], m["moon"], m["atm_model"],
                        m["am_ratio"], m["cd"], m["cr"], m["tol"], m["dt_max_s"], m["method"], embedded,
                        rtol=m.get("rtol"), atol=m.get("atol"), jb_drivers=m.get("jb_drivers"),
                        ground_check=m.get("ground_check", False))


def propagate_batch_final(states, epoch_jd, tof_s, *, ballistic=None, equinoctial=False, gravity_field=None,
                          space_weather=None, ephemeris=None, frame="iau2006", eop=None, **model):
    """Final states of a batch with per-row epoch / duration / ballistics.

    The reference's LightyearSession::integrate_variable_final_into
    (session.rs:2325-2430).  Returns (states_eci [n,6], status [n], steps [n],
    rhs_evals [n]); failed rows are NaN."""
    text, embedded = _field_text(gravity_field)
    ctx = context(text, _batch_cfg(model, embedded), space_weather, ephemeris, frame, eop)
    return ctx.propagate_final(states, epoch_jd, tof_s, ballistic=ballistic, equinoctial=equinoctial)


def propagate_batch_sampled(states, epoch_jd, tof_s, t_eval, *, deltas=False, equinoctial=False,
                            gravity_field=None, space_weather=None, ephemeris=None, frame="iau2006", eop=None,
                            **model):
    """Samples of a batch on one grid; the reference's
    integrate_batch_native_into (batch.rs:247-391) with ``deltas=True``
    (Encke deviations from the initial baseline) or ECI states."""
    text, embedded = _field_text(gravity_field)
    ctx = context(text, _batch_cfg(model, embedded), space_weather, ephemeris, frame, eop)
    return ctx.propagate_sampled(states, epoch_jd, tof_s, t_eval, deltas=deltas, equinoctial=equinoctial)
