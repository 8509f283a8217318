"""Read the reference's Runge-Kutta tableau sources as binary64 numbers.

The reference writes each tableau as Rust constant arrays whose entries are
decimal literals or short constant expressions of them (``35.0 / 384.0 -
5_179.0 / 57_600.0``); Rust evaluates those in IEEE binary64 with
round-to-nearest, one operation at a time, exactly as Python's ``float``
arithmetic does, and parses each literal with correct rounding, as
``float()`` does.  So evaluating the same expressions here gives the same
bits the reference steps with.

Files (inside ``dust_transfer/crates/lightyear_odeint_rs/src/odesolve/tableau``):
``dopri5.rs`` (7 stages), ``dop853.rs`` + ``dop853_coeffs.rs`` (16 stages
truncated to the 12 active ones, with the third-order weights ``E3``),
``vern7.rs`` (10 stages), ``vern9.rs`` (16 stages).  Used by
``make_fixtures.py`` to write ``ref_tableaus.json``.
"""
from __future__ import annotations

import ast
import operator
import re
from pathlib import Path

TABLEAU_DIR = "dust_transfer/crates/lightyear_odeint_rs/src/odesolve/tableau"

_OPS = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv}


def _eval(expr: str) -> float:
    """One Rust f64 constant expression: literals, + - * /, unary minus, parentheses."""
    if "::" in expr:
        raise ValueError(f"named constant in {expr!r}")
    py = expr.replace("_", "")

    def walk(n):
        if isinstance(n, ast.Expression):
            return walk(n.body)
        if isinstance(n, ast.Constant) and isinstance(n.value, (int, float)):
            return float(n.value)
        if isinstance(n, ast.UnaryOp) and isinstance(n.op, ast.USub):
            return -walk(n.operand)
        if isinstance(n, ast.UnaryOp) and isinstance(n.op, ast.UAdd):
            return walk(n.operand)
        if isinstance(n, ast.BinOp) and type(n.op) in _OPS:
            return _OPS[type(n.op)](walk(n.left), walk(n.right))
        raise ValueError(f"unsupported constant expression: {expr!r}")

    return walk(ast.parse(py, mode="eval"))


def _strip_comments(src: str) -> str:
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def _split_top(body: str) -> list[str]:
    """Split on commas that are not inside brackets or parentheses."""
    out, depth, cur = [], 0, []
    for ch in body:
        if ch in "([":
            depth += 1
        elif ch in ")]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    out.append("".join(cur))
    return [t.strip() for t in out if t.strip()]


def _array(src: str, name: str) -> list[float]:
    m = re.search(r"const " + name + r": \[f64; (\d+)\] = \[(.*?)\];", src, re.S)
    if not m:
        raise KeyError(name)
    vals = [_eval(t) for t in _split_top(m.group(2))]
    if len(vals) != int(m.group(1)):
        raise ValueError(f"{name}: {len(vals)} entries, declared {m.group(1)}")
    return vals


def _rows(src: str, stages: int) -> list[list[float]]:
    return [_array(src, f"A{i}") if i else [] for i in range(stages)]


def dopri5(root: Path) -> dict:
    src = _strip_comments((root / TABLEAU_DIR / "dopri5.rs").read_text())
    # rows are named A1..A7 there (A1 empty)
    a = [_array(src, f"A{i + 1}") for i in range(7)]
    return {"c": _array(src, "C"), "a": a, "b": _array(src, "B"), "e": _array(src, "ERR"), "e3": None}


def dop853(root: Path) -> dict:
    src = _strip_comments((root / TABLEAU_DIR / "dop853_coeffs.rs").read_text())
    m = re.search(r"pub const A: Dop853A = \((.*?)\);", src, re.S)
    rows = [[_eval(t) for t in _split_top(r[1:-1])] for r in _split_top(m.group(1))]
    full_c = _array(src.replace("pub const", "const"), "C")
    full_e = _array(src.replace("pub const", "const"), "E")
    b = _array(src.replace("pub const", "const"), "B")
    e3 = _array(src.replace("pub const", "const"), "E3")
    s = 12  # dop853.rs keeps the 12 active stages: A rows A.0..A.10, C/E [0..12)
    if any(v != 0.0 for v in full_e[s:]):
        raise ValueError("dop853: truncated error weights are not zero")
    a = [[]] + [rows[i] for i in range(s - 1)]
    return {"c": full_c[:s], "a": a, "b": b, "e": full_e[:s], "e3": e3}


def verner(root: Path, name: str, stages: int) -> dict:
    src = _strip_comments((root / TABLEAU_DIR / f"{name}.rs").read_text())
    return {"c": _array(src, "C"), "a": _rows(src, stages), "b": _array(src, "B"), "e": _array(src, "ERR"),
            "e3": None}


def read_all(ref_root: str | Path) -> dict:
    root = Path(ref_root)
    return {
        "dopri5": dopri5(root),
        "dop853": dop853(root),
        "vern7": verner(root, "vern7", 10),
        "vern9": verner(root, "vern9", 16),
    }
