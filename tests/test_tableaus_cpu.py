"""Order conditions of the explicit Runge-Kutta tables in ``rk_tableaus.h``.

For every rooted tree t of order |t| <= p the weights of an order-p method
satisfy  sum_i b_i Phi_i(t) = 1 / gamma(t)  (Butcher's conditions; Hairer,
Norsett & Wanner, Solving ODEs I, ch. II.2), and the error weights e of an
embedded pair of error order q satisfy  sum_i e_i Phi_i(t) = 0  for |t| <= q
(both b and b - e are order-q rules) but not for every tree of order q + 1.
The tables are binary64 roundings of the published decimals, so each
condition holds to a tolerance scaled by the size of its terms.
"""
import os
import re
from functools import lru_cache
from pathlib import Path

import numpy as np
import pytest

HEADER = Path(__file__).resolve().parents[1] / "bqp_b200" / "csrc" / "rk_tableaus.h"

# name -> (order, error order, tolerance relative to the sum of |terms|)
PAIRS = {"dopri5": (5, 4, 1e-14), "dop853": (8, 5, 1e-11), "vern7": (7, 6, 1e-11), "vern9": (9, 8, 1e-11)}


def load(name):
    text = HEADER.read_text()

    def arr(suffix):
        m = re.search(rf"bqp_{name}_{suffix}\[\d+\] = \{{(.*?)\}};", text, re.S)
        return np.array([float.fromhex(t) for t in m.group(1).replace(",", " ").split()])

    c, b, e = arr("c"), arr("b"), arr("e")
    s = len(c)
    a = arr("a").reshape(s, s)
    return c, a, b, e


@lru_cache(maxsize=None)
def trees(n):
    """Rooted trees with n vertices, each a sorted tuple of its subtrees."""
    if n == 1:
        return [()]
    out = set()

    def forests(total, min_tree):
        # multisets of trees with `total` vertices, non-decreasing in (order, tree)
        if total == 0:
            yield ()
            return
        for k in range(1, total + 1):
            for t in trees(k):
                key = (k, t)
                if min_tree is not None and key < min_tree:
                    continue
                for rest in forests(total - k, key):
                    yield (t,) + rest

    for f in forests(n - 1, None):
        out.add(tuple(sorted(f, key=lambda t: (size(t), t))))
    return sorted(out, key=lambda t: (len(t), t))


def size(t):
    return 1 + sum(size(u) for u in t)


def gamma(t):
    g = size(t)
    for u in t:
        g *= gamma(u)
    return g


def phi(t, a):
    """Elementary weight vector Phi(t): Phi_i = prod over subtrees u of (A Phi(u))_i."""
    v = np.ones(a.shape[0])
    for u in t:
        v = v * (a @ phi(u, a))
    return v


def test_tree_counts():
    # number of rooted trees of order 1..8 (OEIS A000081)
    assert [len(trees(n)) for n in range(1, 9)] == [1, 1, 2, 4, 9, 20, 48, 115]


@pytest.mark.parametrize("name", sorted(PAIRS))
def test_row_sums(name):
    c, a, b, e = load(name)
    assert np.allclose(a.sum(axis=1), c, rtol=0, atol=1e-13 * max(1.0, np.abs(a).max()))
    assert np.all(np.triu(a) == 0.0)  # explicit


@pytest.mark.parametrize("name", sorted(PAIRS))
def test_order_conditions(name):
    order, order_err, tol = PAIRS[name]
    c, a, b, e = load(name)
    for n in range(1, order + 1):
        for t in trees(n):
            p = phi(t, a)
            got = b @ p
            scale = np.abs(b * p).sum()
            assert abs(got - 1.0 / gamma(t)) <= tol * scale, (name, t, got, 1.0 / gamma(t))
    worst_next = 0.0
    for n in range(1, order_err + 2):
        for t in trees(n):
            p = phi(t, a)
            r = abs(e @ p)
            scale = np.abs(e * p).sum() + np.abs(b * p).sum()
            if n <= order_err:
                assert r <= tol * scale, (name, "error weights", t, r)
            else:
                worst_next = max(worst_next, r * gamma(t))
    assert worst_next > 1e-6, (name, "error estimate vanishes at order", order_err + 1)


@pytest.mark.parametrize("name", sorted(PAIRS))
def test_not_higher_order(name):
    # the stated order is the exact order: some tree of order p + 1 fails
    order, _, _ = PAIRS[name]
    c, a, b, e = load(name)
    worst = max(abs(b @ phi(t, a) - 1.0 / gamma(t)) * gamma(t) for t in trees(order + 1))
    assert worst > 1e-8


def test_vern7_stage_one_pin():
    # the reference pins Vern7's second stage bit for bit
    # (odesolve/tableau/vern7.rs:140-152): c1 = a10 = 0.005, b1 = err1 = 0
    c, a, b, e = load("vern7")
    assert c[1] == 0.005 and a[1, 0] == 0.005
    assert b[1] == 0.0 and e[1] == 0.0
    assert c[-1] == 1.0 and np.all(a[-1, 7:] == 0.0)  # error stage built on stages 0-6


# ---------------------------------------------------------------------------
# Bit equality with the reference's own tables.  tests/golden/ref_tableaus.json
# holds every entry of the reference's odesolve/tableau/{dopri5, dop853 +
# dop853_coeffs, vern7, vern9}.rs as binary64 (make_fixtures.py evaluates the
# Rust constant expressions); the product header (generated from published
# fractions and constants) and the oracle's own header (generated from that
# fixture) must both carry exactly those bits, so neither side can share a
# wrong weight with the other unnoticed.  This pins the embedded error
# weights e and DOP853's third-order e3, which the order conditions above
# only constrain up to the error order.

REF_TABLES = Path(__file__).resolve().parent / "golden" / "ref_tableaus.json"
ORACLE_HEADER = Path(__file__).resolve().parents[1] / "oracle" / "ref_tableaus.h"


def header_arrays(path, prefix, name):
    text = path.read_text()
    out = {}
    for key in ("c", "a", "b", "e", "e3"):
        m = re.search(rf"{prefix}_{name}_{key}\[\d+\] = \{{(.*?)\}};", text, re.S)
        out[key] = None if m is None else [float.fromhex(t) for t in m.group(1).replace(",", " ").split()]
    return out


def fixture_arrays(name):
    import json
    t = json.loads(REF_TABLES.read_text())["tables"][name]
    s = t["stages"]
    flat = []
    for row in t["a"]:
        flat += [float.fromhex(x) for x in row] + [0.0] * (s - len(row))
    conv = lambda v: None if v is None else [float.fromhex(x) for x in v]  # noqa: E731
    return {"c": conv(t["c"]), "a": flat, "b": conv(t["b"]), "e": conv(t["e"]), "e3": conv(t["e3"])}


def bits(v):
    return [float(x).hex() for x in v]


@pytest.mark.parametrize("name", sorted(PAIRS))
@pytest.mark.parametrize("side", ["product", "oracle"])
def test_tables_bit_equal_to_reference(name, side):
    ref = fixture_arrays(name)
    got = header_arrays(HEADER, "bqp", name) if side == "product" else header_arrays(ORACLE_HEADER, "ref", name)
    for key in ("c", "a", "b", "e", "e3"):
        if ref[key] is None:
            assert got[key] is None, (name, key)
            continue
        assert got[key] is not None and len(got[key]) == len(ref[key]), (side, name, key)
        diff = [i for i, (x, y) in enumerate(zip(bits(got[key]), bits(ref[key]))) if x != y]
        assert not diff, (side, name, key, diff[:5])


def test_reference_shapes():
    # stage counts and the DOP853 truncation to its 12 active stages (dop853.rs:1-97)
    import json
    t = json.loads(REF_TABLES.read_text())["tables"]
    assert {k: v["stages"] for k, v in t.items()} == {"dopri5": 7, "dop853": 12, "vern7": 10, "vern9": 16}
    assert t["dop853"]["e3"] is not None and all(t[k]["e3"] is None for k in ("dopri5", "vern7", "vern9"))
    # Vern9's last stage is built on stages 0-12 only (vern9.rs:213-227)
    assert len(t["vern9"]["a"][15]) == 13 and len(t["vern7"]["a"][9]) == 7


@pytest.mark.skipif(not os.environ.get("BQP_REFERENCE_ROOT"), reason="BQP_REFERENCE_ROOT not set")
def test_fixture_matches_reference_sources():
    # re-evaluate the reference's sources when its tree is at hand
    import sys
    sys.path.insert(0, str(REF_TABLES.parent))
    import rust_tableaus
    tabs = rust_tableaus.read_all(os.environ["BQP_REFERENCE_ROOT"])
    for name in PAIRS:
        ref = fixture_arrays(name)
        t = tabs[name]
        s = len(t["c"])
        flat = [x for row in t["a"] for x in row + [0.0] * (s - len(row))]
        assert bits(flat) == bits(ref["a"]) and bits(t["b"]) == bits(ref["b"]) and bits(t["e"]) == bits(ref["e"])
        assert bits(t["c"]) == bits(ref["c"])
        assert (t["e3"] is None) == (ref["e3"] is None)
        if t["e3"] is not None:
            assert bits(t["e3"]) == bits(ref["e3"])
