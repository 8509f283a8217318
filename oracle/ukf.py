"""CPU restatement of the reference's sigma-point (UKF) transform.

TEST INFRASTRUCTURE ONLY: tests/ use this module as the checker of the
device sigma-point generation and recombination (bqp_sigma_propagate).

Follows dust_transfer/crates/dust_ukf_rs/src/lib.rs:
* julier_offsets      -- Julier's n + 2 simplex recursion at W0 = 0 with the
                         centre point dropped (lib.rs:155-200), weights 1/7
                         (lib.rs:69-78)
* repair_to_psd       -- eigenvalues below 1e-12 raised to 1e-12, None when
                         none was below (lib.rs:202-240)
* get_sigmas          -- x_i = mean + L xi_i, L = chol(P), repair on failure
                         (lib.rs:247-275)
* rebuild_mean_covar  -- weighted mean, weighted outer products, then
                         symmetrised (lib.rs:277-312); the 13-point set sums
                         deviations about its centre point instead
and, for the 13-point set the reference retired, the published scaled
unscented transform of Wan & van der Merwe (2000): lambda = alpha^2 (n +
kappa) - n, L = chol((n + lambda) P), x_0 = mean, x_{1+i} = mean + L e_i,
x_{7+i} = mean - L e_i, Wm_0 = lambda/(n+lambda), Wc_0 = Wm_0 + 1 - alpha^2 +
beta, W_i = 1/(2(n+lambda)).
"""
from __future__ import annotations

import numpy as np

N = 6


def julier_offsets() -> np.ndarray:
    w1 = 1.0 / (N + 1.0)
    seq = np.zeros((N + 2, N))
    seq[1, 0] = -1.0 / np.sqrt(2.0 * w1)
    seq[2, 0] = 1.0 / np.sqrt(2.0 * w1)
    jf = 1.0
    for j in range(2, N + 1):
        jf += 1.0
        step = 1.0 / np.sqrt(jf * (jf + 1.0) * w1)
        seq[1:j + 1, j - 1] = -step
        seq[j + 1, :] = 0.0
        seq[j + 1, j - 1] = jf * step
    return seq[1:].copy()


def weights(sigma_set="julier7", alpha=1e-3, beta=2.0, kappa=0.0):
    if sigma_set == "julier7":
        w = np.full(N + 1, 1.0 / (N + 1.0))
        return w, w.copy(), 1.0
    lam = alpha * alpha * (N + kappa) - N
    c = N + lam
    wm = np.full(2 * N + 1, 1.0 / (2.0 * c))
    wc = wm.copy()
    wm[0] = lam / c
    wc[0] = lam / c + (1.0 - alpha * alpha + beta)
    return wm, wc, c


def _chol(p):
    # nalgebra's Cholesky::new declines a non-positive or non-finite pivot
    l = np.zeros((N, N))
    for j in range(N):
        s = p[j, j] - np.dot(l[j, :j], l[j, :j])
        if not (s > 0.0) or not np.isfinite(s):
            return None
        d = np.sqrt(s)
        l[j, j] = d
        for i in range(j + 1, N):
            l[i, j] = (p[i, j] - np.dot(l[i, :j], l[j, :j])) / d
    return l


def repair_to_psd(p):
    if not np.isfinite(p).all():
        return None  # NaN eigenvalues compare false with the floor: nothing floored
    w, v = np.linalg.eigh(p)
    floored = w < 1e-12
    if not floored.any():
        return None
    w = np.where(floored, 1e-12, w)
    return (v * w) @ v.T


def get_sigmas(mean, cov, sigma_set="julier7", alpha=1e-3, beta=2.0, kappa=0.0):
    """Sigma points [S][6], or None when the covariance cannot be factorised."""
    _, _, scale = weights(sigma_set, alpha, beta, kappa)
    p = np.asarray(cov, dtype=np.float64).reshape(N, N) * scale
    l = _chol(p)
    if l is None:
        r = repair_to_psd(p)
        l = None if r is None else _chol(r)
        if l is None:
            return None
    m = np.asarray(mean, dtype=np.float64)
    if sigma_set == "julier7":
        return np.array([m + l @ xi for xi in julier_offsets()])
    return np.array([m] + [m + l[:, i] for i in range(N)] + [m - l[:, i] for i in range(N)])


def rebuild_mean_covar(sigmas, wm, wc):
    s = np.asarray(sigmas, dtype=np.float64)
    if s.shape[0] == 2 * N + 1:
        # scaled set: the same moments from deviations about the centre point
        # (the device's evaluation order; Wm_0 ~ -1/alpha^2 makes the plain
        # sum ill-conditioned)
        dm = np.zeros(N)
        for i in range(1, s.shape[0]):
            dm += wm[i] * (s[i] - s[0])
        cov = np.zeros((N, N))
        for i in range(s.shape[0]):
            d = (s[i] - s[0]) - dm
            cov += wc[i] * np.outer(d, d)
        return s[0] + dm, 0.5 * (cov + cov.T)
    mean = np.zeros(N)
    for i in range(s.shape[0]):
        mean += wm[i] * s[i]
    cov = np.zeros((N, N))
    for i in range(s.shape[0]):
        d = s[i] - mean
        cov += wc[i] * np.outer(d, d)
    return mean, 0.5 * (cov + cov.T)
