"""Sigma-point sets on the CPU: the restatement and the library's host-side
weights against the reference's literal Julier offsets, and the unscented
transform's moment properties."""
import json
import struct
from pathlib import Path

import numpy as np
import pytest

from bqp_b200 import _native as N
from bqp_b200 import workloads
from oracle import ukf as U

GOLDEN = Path(__file__).resolve().parent / "golden" / "julier7_offsets.json"


def bits(v):
    return struct.pack(">d", float(v)).hex()


def test_julier_offsets_bit_equal_to_reference_literals():
    g = json.loads(GOLDEN.read_text())
    ref = np.array(g["offsets"])
    assert ref.shape == (7, 6)
    ours = U.julier_offsets()
    assert [[bits(v) for v in r] for r in ours] == g["bits"]
    p, wm, wc, off = N.sigma_weights("julier7")
    assert p == 7
    assert [[bits(v) for v in r] for r in off] == g["bits"]
    assert (wm == 1.0 / 7.0).all() and (wc == 1.0 / 7.0).all()


def test_merwe_weights_match_published_formulas():
    for alpha, beta, kappa in [(1e-3, 2.0, 0.0), (0.5, 2.0, 1.0), (1.0, 0.0, 3.0)]:
        p, wm, wc, off = N.sigma_weights("merwe13", alpha, beta, kappa)
        owm, owc, _ = U.weights("merwe13", alpha, beta, kappa)
        assert p == 13
        assert np.allclose(wm, owm, rtol=1e-15, atol=0) and np.allclose(wc, owc, rtol=1e-15, atol=0)
        assert abs(wm.sum() - 1.0) < 1e-9 * max(1.0, abs(wm[0]))
    with pytest.raises(N.NativeError):
        N.sigma_weights("merwe13", 0.0, 2.0, 0.0)


@pytest.mark.parametrize("sigma_set", ["julier7", "merwe13"])
def test_unscented_transform_reproduces_linear_moments(sigma_set):
    means, covs = workloads.ukf_objects(16, seed=2)
    wm, wc, _ = U.weights(sigma_set)
    for m, c in zip(means, covs):
        s = U.get_sigmas(m, c, sigma_set)
        mm, cc = U.rebuild_mean_covar(s, wm, wc)
        assert np.allclose(mm, m, rtol=0, atol=1e-9 * np.abs(m).max())
        assert np.linalg.norm(cc - c) <= 1e-6 * np.linalg.norm(c)


def test_repair_floors_eigenvalues_like_the_reference():
    c = np.diag([1.0, 1.0, 1.0, 1e-6, 1e-6, -1e-9])  # one negative eigenvalue
    assert U._chol(c) is None
    r = U.repair_to_psd(c)
    assert np.linalg.eigvalsh(r).min() >= 1e-12 * (1 - 1e-9)
    assert U.get_sigmas(np.zeros(6), c) is not None
    # nothing below the floor -> no repair -> failure (lib.rs:224-226)
    assert U.repair_to_psd(np.diag([1.0] * 6)) is None
    assert U.get_sigmas(np.zeros(6), np.full((6, 6), np.nan)) is None
