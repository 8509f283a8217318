"""Seeded synthetic inputs of the benchmark configurations.

No public dataset is involved: every input is generated here with
``numpy.random.default_rng`` so the GPU path, the CPU oracle and the CPU
baseline all see identical arrays.

* ``synthetic_field(order, seed)``: normalised coefficients, C20 = -4.84165e-4,
  every other C_nm, S_nm ~ N(0, (1e-5/n^2)^2) for n >= 2 (S_n0 = 0, degree 1
  zero) -- the "synthetic N x N normalised field / Kaula rule" of the configs,
  written as ``deg ord C S`` text (the reference loader's format).
* ``leo_states(n, seed)``: altitude (a - R_E) U[400, 1200] km, e U[0, 0.02],
  i U[0, 98] deg, RAAN / argp / mean anomaly U[0, 360) deg; the mean anomaly
  is converted to the true anomaly, then to ECI.
* ``mixed_states``: the uneven-batch mix (60% LEO, 20% MEO, 10% GEO, 10% HEO)
  with log-uniform durations.
"""
from __future__ import annotations

import numpy as np

RE_KM = 6378.137
MU_KM3_S2 = 398600.4415  # the reference's mu (satpy_core/src/lib.rs:74)
EPOCH_JD = 2460310.5  # 2024-01-01T00:00 UTC, the reference smoke test's epoch


def synthetic_field(order: int, seed: int | None = None) -> str:
    if seed is None:
        seed = 12345 + order
    rng = np.random.default_rng(seed)
    lines = ["# synthetic normalised field: C20 = -4.84165e-4, C/S ~ N(0, (1e-5/n^2)^2)"]
    for n in range(2, order + 1):
        sig = 1e-5 / (n * n)
        c = rng.normal(0.0, sig, n + 1)
        s = rng.normal(0.0, sig, n + 1)
        s[0] = 0.0
        if n == 2:
            c[0] = -4.84165e-4
        for m in range(n + 1):
            lines.append(f"{n} {m} {float(c[m])!r} {float(s[m])!r}")
    return "\n".join(lines) + "\n"


def mean_to_true(M: np.ndarray, e: np.ndarray) -> np.ndarray:
    E = M.copy()
    for _ in range(50):
        E = E - (E - e * np.sin(E) - M) / (1.0 - e * np.cos(E))
    return 2.0 * np.arctan2(np.sqrt(1 + e) * np.sin(E / 2), np.sqrt(1 - e) * np.cos(E / 2))


def kep_to_eci(kep: np.ndarray, mu: float = MU_KM3_S2) -> np.ndarray:
    """[a km, e, i, RAAN, argp, true anomaly (deg)] -> ECI [n][6]: the
    perifocal position and velocity rotated by R3(-RAAN) R1(-i) R3(-argp).
    Plain numpy, so generating a workload loads no native library."""
    kep = np.asarray(kep, dtype=np.float64).reshape(-1, 6)
    a, e = kep[:, 0], kep[:, 1]
    inc, raan, argp, nu = (np.radians(kep[:, k]) for k in (2, 3, 4, 5))
    p = a * (1.0 - e * e)
    cn, sn = np.cos(nu), np.sin(nu)
    r = p / (1.0 + e * cn)
    sp = np.sqrt(mu / p)
    xp, yp = r * cn, r * sn
    vxp, vyp = -sp * sn, sp * (e + cn)
    cO, sO, cw, sw, ci, si = np.cos(raan), np.sin(raan), np.cos(argp), np.sin(argp), np.cos(inc), np.sin(inc)
    r00, r01 = cO * cw - sO * sw * ci, -cO * sw - sO * cw * ci
    r10, r11 = sO * cw + cO * sw * ci, -sO * sw + cO * cw * ci
    r20, r21 = sw * si, cw * si
    out = np.stack([r00 * xp + r01 * yp, r10 * xp + r11 * yp, r20 * xp + r21 * yp,
                    r00 * vxp + r01 * vyp, r10 * vxp + r11 * vyp, r20 * vxp + r21 * vyp], axis=1)
    bad = ~((a > 0.0) & (e >= 0.0) & (e < 1.0))
    out[bad] = np.nan
    return np.ascontiguousarray(out)


def kep_states(a, e, i_deg, raan_deg, argp_deg, M_deg) -> np.ndarray:
    nu = np.degrees(mean_to_true(np.radians(M_deg), e)) % 360.0
    kep = np.stack([a, e, i_deg, raan_deg, argp_deg, nu], axis=1)
    return kep_to_eci(kep)


def leo_states(n: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    alt = rng.uniform(400.0, 1200.0, n)
    e = rng.uniform(0.0, 0.02, n)
    inc = rng.uniform(0.0, 98.0, n)
    raan = rng.uniform(0.0, 360.0, n)
    argp = rng.uniform(0.0, 360.0, n)
    M = rng.uniform(0.0, 360.0, n)
    return kep_states(RE_KM + alt, e, inc, raan, argp, M)


def leo_ballistics(n: int, seed: int = 0) -> np.ndarray:
    """(A/m U[0.005, 0.05] m^2/kg, Cd = 2.2) per row."""
    rng = np.random.default_rng(seed + 7919)
    am = rng.uniform(0.005, 0.05, n)
    return np.stack([am, np.full(n, 2.2)], axis=1)


def mixed_states(n: int, seed: int = 0):
    """60% LEO / 20% MEO (a U[20000, 27000]) / 10% GEO / 10% HEO (e U[0.5, 0.75],
    perigee altitude 500 km); durations log-uniform 1 h .. 30 d.
    Returns (states [n,6], durations_s [n], is_low [n]): is_low marks the
    orbits whose perigee is below 2000 km (LEO and HEO), where drag applies."""
    rng = np.random.default_rng(seed)
    kind = rng.choice(4, size=n, p=[0.6, 0.2, 0.1, 0.1])
    a = np.empty(n)
    e = np.empty(n)
    a[kind == 0] = RE_KM + rng.uniform(400.0, 1200.0, (kind == 0).sum())
    e[kind == 0] = rng.uniform(0.0, 0.02, (kind == 0).sum())
    a[kind == 1] = rng.uniform(20000.0, 27000.0, (kind == 1).sum())
    e[kind == 1] = rng.uniform(0.0, 0.02, (kind == 1).sum())
    a[kind == 2] = 42164.0 + rng.uniform(-50.0, 50.0, (kind == 2).sum())
    e[kind == 2] = rng.uniform(0.0, 0.001, (kind == 2).sum())
    eh = rng.uniform(0.5, 0.75, (kind == 3).sum())
    e[kind == 3] = eh
    a[kind == 3] = (RE_KM + 500.0) / (1.0 - eh)
    inc = rng.uniform(0.0, 98.0, n)
    inc[kind == 2] = rng.uniform(0.0, 1.0, (kind == 2).sum())
    raan = rng.uniform(0.0, 360.0, n)
    argp = rng.uniform(0.0, 360.0, n)
    M = rng.uniform(0.0, 360.0, n)
    states = kep_states(a, e, inc, raan, argp, M)
    dur = np.exp(rng.uniform(np.log(3600.0), np.log(30 * 86400.0), n))
    return states, dur, a * (1.0 - e) - RE_KM < 2000.0


def mixed_ballistics(is_low, seed: int = 0) -> np.ndarray:
    """Per-row (A/m, Cd) of the mixed workload: A/m U[0.005, 0.05] m^2/kg
    where drag applies (perigee below 2000 km), 0 (no drag call) elsewhere."""
    b = leo_ballistics(len(is_low), seed=seed)
    b[~np.asarray(is_low), 0] = 0.0
    return b


def ukf_objects(n: int, seed: int = 0):
    """Means and covariances of the sigma-point workload: LEO means (the
    distributions of leo_states) and random SPD covariances with position
    sigmas U[10, 1000] m and velocity sigmas U[0.01, 1] m/s, correlated
    through a random correlation matrix.  Returns (mean[n][6] km, km/s,
    cov[n][6][6] km^2 ...)."""
    rng = np.random.default_rng(seed + 7919)
    means = leo_states(n, seed=seed)
    sig = np.concatenate([rng.uniform(10.0, 1000.0, (n, 3)) * 1e-3, rng.uniform(0.01, 1.0, (n, 3)) * 1e-3], axis=1)
    covs = np.empty((n, 6, 6))
    for i in range(n):
        a = rng.normal(size=(6, 6))
        c = a @ a.T + 6.0 * np.eye(6)
        d = 1.0 / np.sqrt(np.diag(c))
        corr = c * d[:, None] * d[None, :]
        covs[i] = corr * sig[i][:, None] * sig[i][None, :]
    return means, covs


def orbit_period_s(states) -> np.ndarray:
    """Two-body period of each ECI state (mu = 398600.4415 km^3/s^2)."""
    s = np.asarray(states, dtype=np.float64).reshape(-1, 6)
    r = np.linalg.norm(s[:, :3], axis=1)
    v2 = np.einsum("ij,ij->i", s[:, 3:], s[:, 3:])
    mu = 398600.4415
    a = 1.0 / (2.0 / r - v2 / mu)
    return 2.0 * np.pi * np.sqrt(a ** 3 / mu)
