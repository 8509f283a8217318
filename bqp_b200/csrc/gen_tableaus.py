"""Generate ``rk_tableaus.h``: the Butcher tableaus of the two explicit RK pairs.

* DOPRI5(4): Dormand & Prince (1980), 7 stages, FSAL, written here as exact
  fractions (the same fractions as the reference's
  ``odesolve/tableau/dopri5.rs``).
* DOP853: Hairer, Norsett & Wanner's ``dop853`` (Solving ODEs I, 2nd ed.),
  truncated to its 12 active stages with the 5th-order error weights ``E5`` and
  the 3rd-order weights ``E3 = B - BHH``.  The numbers are taken from SciPy's
  published copy of Hairer's coefficients (``scipy.integrate._ivp.
  dop853_coefficients``), which carries the same decimal constants as the
  reference's ``odesolve/tableau/dop853_coeffs.rs``.

* Vern7 and Vern9: Verner's 7(6) and 9(8) "numerically optimal" pairs (J.H.
  Verner, Numerical Algorithms 53 (2010) 383-396), 10 and 16 stages, not
  FSAL.  Vern7's tenth stage (c = 1, built on stages 0-6) serves only the
  error estimate; Vern9's stages 14 and 15 both sit at c = 1, the second built
  on stages 0-12 for the error estimate only.  Their published decimal
  constants are read from the reference's ``odesolve/tableau/vern7.rs`` and
  ``vern9.rs`` when the header is generated (the reference tree is needed
  only then), so both sides step with the same binary64 numbers.

Values are emitted as C99 hex-float literals so the header is bit-exact.
Run: ``python bqp_b200/csrc/gen_tableaus.py REFERENCE_ROOT`` (or set
``BQP_REFERENCE_ROOT``; rewrites the header in place).
"""
import os
import re
import sys
from fractions import Fraction as F
from pathlib import Path

import numpy as np


def dopri5():
    c = [F(0), F(1, 5), F(3, 10), F(4, 5), F(8, 9), F(1), F(1)]
    a = [
        [],
        [F(1, 5)],
        [F(3, 40), F(9, 40)],
        [F(44, 45), F(-56, 15), F(32, 9)],
        [F(19372, 6561), F(-25360, 2187), F(64448, 6561), F(-212, 729)],
        [F(9017, 3168), F(-355, 33), F(46732, 5247), F(49, 176), F(-5103, 18656)],
        [F(35, 384), F(0), F(500, 1113), F(125, 192), F(-2187, 6784), F(11, 84)],
    ]
    b = [F(35, 384), F(0), F(500, 1113), F(125, 192), F(-2187, 6784), F(11, 84), F(0)]
    bhat = [F(5179, 57600), F(0), F(7571, 16695), F(393, 640), F(-92097, 339200),
            F(187, 2100), F(1, 40)]
    # error weights are formed in binary64 as b - bhat, term by term, which is how
    # the reference's constant table evaluates them
    err = [float(bi) - float(bh) for bi, bh in zip(b, bhat)]
    err[6] = -1.0 / 40.0
    af = [[float(x) for x in row] for row in a]
    return [float(x) for x in c], af, [float(x) for x in b], err, None


def dop853():
    import scipy.integrate._ivp.dop853_coefficients as d
    s = 12
    c = [float(x) for x in d.C[:s]]
    a = [[float(d.A[i, j]) for j in range(i)] for i in range(s)]
    b = [float(x) for x in d.B[:s]]
    e5 = [float(x) for x in d.E5[:s]]
    e3 = [float(x) for x in d.E3[:s]]
    return c, a, b, e5, e3


def verner(ref_root: str, name: str, stages: int):
    """Arrays C, A0..A{stages-1}, B and ERR of ``tableau/<name>.rs`` (Rust
    array literals of decimal constants with ``_`` digit separators)."""
    src = (Path(ref_root) / f"dust_transfer/crates/lightyear_odeint_rs/src/odesolve/tableau/{name}.rs").read_text()
    src = re.sub(r"//[^\n]*", "", src)  # comments may hold numbers

    def arr(key):
        m = re.search(r"const " + key + r": \[f64; (\d+)\] = \[(.*?)\];", src, re.S)
        vals = [float(t.replace("_", "")) for t in re.findall(r"-?[0-9][0-9_]*\.[0-9_]*(?:e-?[0-9]+)?", m.group(2))]
        assert len(vals) == int(m.group(1)), (name, key)
        return vals

    c = arr("C")
    a = [arr(f"A{i}") if i else [] for i in range(stages)]
    b = arr("B")
    e = arr("ERR")
    assert len(c) == len(b) == len(e) == stages
    return c, a, b, e, None


def vern7(ref_root: str):
    return verner(ref_root, "vern7", 10)


def vern9(ref_root: str):
    return verner(ref_root, "vern9", 16)


def hexf(x: float) -> str:
    if x == 0.0:
        return "0.0"
    return float(x).hex()


def emit(name, tab, order, order_err, fsal):
    c, a, b, e, e3 = tab
    s = len(c)
    lines = [f"// {name}: {s} stages, order {order}, error order {order_err}"]
    lines.append(f"#define BQP_{name.upper()}_STAGES {s}")
    lines.append(f"#define BQP_{name.upper()}_ORDER_ERR {order_err}")
    lines.append(f"#define BQP_{name.upper()}_FSAL {1 if fsal else 0}")
    lines.append(f"BQP_TAB_CONST double bqp_{name}_c[{s}] = {{" + ", ".join(hexf(x) for x in c) + "};")
    flat = []
    for i in range(s):
        row = a[i] + [0.0] * (s - len(a[i]))
        flat.extend(row)
    lines.append(f"BQP_TAB_CONST double bqp_{name}_a[{s * s}] = {{")
    for i in range(s):
        lines.append("  " + ", ".join(hexf(x) for x in flat[i * s:(i + 1) * s]) + ",")
    lines.append("};")
    lines.append(f"BQP_TAB_CONST double bqp_{name}_b[{s}] = {{" + ", ".join(hexf(x) for x in b) + "};")
    lines.append(f"BQP_TAB_CONST double bqp_{name}_e[{s}] = {{" + ", ".join(hexf(x) for x in e) + "};")
    if e3 is not None:
        lines.append(f"BQP_TAB_CONST double bqp_{name}_e3[{s}] = {{" + ", ".join(hexf(x) for x in e3) + "};")
    return "\n".join(lines) + "\n"


def main(ref_root: str | None = None):
    ref_root = ref_root or os.environ.get("BQP_REFERENCE_ROOT")
    if not ref_root:
        raise SystemExit("usage: gen_tableaus.py REFERENCE_ROOT (or set BQP_REFERENCE_ROOT)")
    out = Path(__file__).with_name("rk_tableaus.h")
    text = [
        "// Generated by gen_tableaus.py -- do not edit by hand.",
        "// Explicit Runge-Kutta pairs used by the propagator (see gen_tableaus.py",
        "// for the published sources of each table).",
        "#pragma once",
        "#ifndef BQP_TAB_CONST",
        "#define BQP_TAB_CONST static const",
        "#endif",
        "",
        emit("dopri5", dopri5(), 5, 4, True),
        emit("dop853", dop853(), 8, 5, False),
        emit("vern7", vern7(ref_root), 7, 6, False),
        emit("vern9", vern9(ref_root), 9, 8, False),
    ]
    out.write_text("\n".join(text))
    # sanity: row sums equal nodes
    for name, tab in (("dopri5", dopri5()), ("dop853", dop853()), ("vern7", vern7(ref_root)),
                      ("vern9", vern9(ref_root))):
        c, a, *_ = tab
        for i, row in enumerate(a):
            # binary64 constants: the sum is exact only to the rounding of
            # its largest terms (Vern7's error stage reaches |a| ~ 187)
            assert abs(sum(row) - c[i]) <= 1e-15 * max([1.0] + [abs(x) for x in row]) * max(1, len(row)), (name, i)
    print("wrote", out)


if __name__ == "__main__":
    main(*sys.argv[1:])
