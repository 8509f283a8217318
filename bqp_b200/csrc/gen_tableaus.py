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

* Vern7: Verner's 7(6) "numerically optimal" pair (J.H. Verner, Numerical
  Algorithms 53 (2010) 383-396), 10 stages, not FSAL; the tenth stage (c = 1,
  built on stages 0-6) serves only the error estimate.  Its published decimal
  constants are read from the reference's ``odesolve/tableau/vern7.rs`` when
  the header is generated (the reference tree is needed only then), so both
  sides step with the same binary64 numbers.

Values are emitted as C99 hex-float literals so the header is bit-exact.
Run: ``python bqp_b200/csrc/gen_tableaus.py [REFERENCE_ROOT]`` (rewrites the
header in place).
"""
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


def vern7(ref_root: str):
    src = (Path(ref_root) / "dust_transfer/crates/lightyear_odeint_rs/src/odesolve/tableau/vern7.rs").read_text()

    def arr(name):
        m = re.search(r"const " + name + r": \[f64; \d+\] = \[(.*?)\];", src, re.S)
        return [float(t.replace("_", "")) for t in re.findall(r"-?[0-9][0-9_]*\.[0-9_]*(?:e-?[0-9]+)?", m.group(1))]

    c = arr("C")
    a = [arr(f"A{i}") if i else [] for i in range(10)]
    b = arr("B")
    e = arr("ERR")
    return c, a, b, e, None


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


def main(ref_root: str = "/root/reference"):
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
    ]
    out.write_text("\n".join(text))
    # sanity: row sums equal nodes
    for name, tab in (("dopri5", dopri5()), ("dop853", dop853()), ("vern7", vern7(ref_root))):
        c, a, *_ = tab
        for i, row in enumerate(a):
            # binary64 constants: the sum is exact only to the rounding of
            # its largest terms (Vern7's error stage reaches |a| ~ 187)
            assert abs(sum(row) - c[i]) <= 1e-15 * max([1.0] + [abs(x) for x in row]) * max(1, len(row)), (name, i)
    print("wrote", out)


if __name__ == "__main__":
    main(*sys.argv[1:])
