"""Write ``oracle/ref_tableaus.h``: the oracle's own copy of the reference's
Runge-Kutta tables (test infrastructure, not product code).

The numbers come from ``tests/golden/ref_tableaus.json``, which
``tests/golden/make_fixtures.py`` evaluates from the reference's tableau
sources (``lightyear_odeint_rs/src/odesolve/tableau/*.rs``) bit for bit.  The
product's ``bqp_b200/csrc/rk_tableaus.h`` is generated separately, from the
published fractions and constants; ``tests/test_tableaus_cpu.py`` checks both
against the fixture, so a wrong weight on either side fails a test instead of
being shared by the two.

Run: ``python oracle/gen_ref_tableaus.py`` (rewrites the header in place).
"""
import json
from pathlib import Path

HERE = Path(__file__).resolve().parent
FIXTURE = HERE.parent / "tests" / "golden" / "ref_tableaus.json"
OUT = HERE / "ref_tableaus.h"


def lit(h: str) -> str:
    v = float.fromhex(h)
    return "0.0" if v == 0.0 and not h.startswith("-") else h


def main() -> None:
    tabs = json.loads(FIXTURE.read_text())["tables"]
    lines = ["// Generated by oracle/gen_ref_tableaus.py from tests/golden/ref_tableaus.json",
             "// (the reference's odesolve/tableau/*.rs, evaluated bit for bit). Oracle only.",
             "#pragma once", ""]
    for name, t in tabs.items():
        s = t["stages"]
        lines.append(f"// {name}: {s} stages; a is s x s row-major, rows zero-padded")
        lines.append(f"static const double ref_{name}_c[{s}] = {{{', '.join(lit(x) for x in t['c'])}}};")
        lines.append(f"static const double ref_{name}_a[{s * s}] = {{")
        for row in t["a"]:
            full = [lit(x) for x in row] + ["0.0"] * (s - len(row))
            lines.append("  " + ", ".join(full) + ",")
        lines.append("};")
        for key in ("b", "e", "e3"):
            if t[key] is not None:
                lines.append(f"static const double ref_{name}_{key}[{s}] = {{{', '.join(lit(x) for x in t[key])}}};")
        lines.append("")
    OUT.write_text("\n".join(lines))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
