"""Generate ``iau2000a_tables.h``: the published series of the IAU 2006/2000A
CIO-based frame chain.

* IAU 2000A nutation (Mathews, Herring & Buffett 2002; IERS Conventions 2003,
  chapter 5, tables 5.3a/5.3b): 678 luni-solar terms, each with the five
  Delaunay multipliers and the (sp, spt, cp, ce, cet, se) amplitudes in units
  of 0.1 microarcsecond, and 687 planetary terms with 13 multipliers and
  integer amplitudes.
* The series part of the IAU 2006 CIO locator s + XY/2 (IERS Conventions
  2010, table 5.2d), in arcseconds: the terms of t^0 (33), t^1 (3), t^2 (25),
  t^3 (4) and t^4 (1), each with eight fundamental-argument multipliers.

The numbers are the published tables, in the order of ERFA's ``nut00a.c`` and
``s06.c``.  They are read from the reference's ``satpy_core/src/frame_time/
tables.rs`` when the header is generated (the reference tree is needed only
then), so both sides sum the same binary64 values in the same order.  Values
are emitted as C99 hex-float literals so the header is bit-exact.

Run: ``python bqp_b200/csrc/gen_iau_tables.py REFERENCE_ROOT`` (or set
``BQP_REFERENCE_ROOT``; rewrites the header in place).
"""
import os
import re
import sys
from pathlib import Path

TABLES = "dust_transfer/crates/satpy_core/src/frame_time/tables.rs"


def num(text):
    return float(text.replace("_", ""))


def parse(src):
    ls, pl, s06 = [], [], {}
    for m in re.finditer(r"NutLs \{ n: \[([^\]]*)\], sp: ([^,]+), spt: ([^,]+), cp: ([^,]+), "
                         r"ce: ([^,]+), cet: ([^,]+), se: ([^ ]+) \}", src):
        ls.append(([int(v) for v in m.group(1).split(",")], [num(m.group(k)) for k in range(2, 8)]))
    for m in re.finditer(r"NutPl \{ n: \[([^\]]*)\], sp: ([^,]+), cp: ([^,]+), se: ([^,]+), "
                         r"ce: ([^ ]+) \}", src):
        pl.append(([int(v) for v in m.group(1).split(",")], [int(m.group(k)) for k in range(2, 6)]))
    for blk in re.finditer(r"pub static (S06_S\d): \[CioTerm; (\d+)\] = \[(.*?)\];", src, re.S):
        terms = []
        for m in re.finditer(r"CioTerm \{ n: \[([^\]]*)\], s: ([^,]+), c: ([^ ]+) \}", blk.group(3)):
            terms.append(([int(v) for v in m.group(1).split(",")], [num(m.group(2)), num(m.group(3))]))
        assert len(terms) == int(blk.group(2)), blk.group(1)
        s06[blk.group(1)] = terms
    assert len(ls) == 678 and len(pl) == 687, (len(ls), len(pl))
    assert sorted(s06) == ["S06_S0", "S06_S1", "S06_S2", "S06_S3", "S06_S4"]
    return ls, pl, s06


def hexf(x):
    return float(x).hex()


def emit(ls, pl, s06):
    out = ["// Generated by gen_iau_tables.py from the published IAU 2000A nutation and",
           "// IAU 2006 CIO-locator series; do not edit.",
           "#pragma once",
           "#include <cstdint>",
           "",
           "namespace bqp { namespace iau {",
           "",
           "struct NutLs { int8_t n[5]; double sp, spt, cp, ce, cet, se; };",
           "struct NutPl { int8_t n[13]; int32_t sp, cp, se, ce; };",
           "struct CioTerm { int8_t n[8]; double s, c; };",
           "",
           f"constexpr int kNutLs = {len(ls)};",
           f"constexpr int kNutPl = {len(pl)};",
           "",
           "static const NutLs kNutLsTab[kNutLs] = {"]
    for n, a in ls:
        out.append("    {{%s}, %s}," % (", ".join(map(str, n)), ", ".join(hexf(v) for v in a)))
    out.append("};")
    out.append("")
    out.append("static const NutPl kNutPlTab[kNutPl] = {")
    for n, a in pl:
        out.append("    {{%s}, %s}," % (", ".join(map(str, n)), ", ".join(map(str, a))))
    out.append("};")
    for name in sorted(s06):
        terms = s06[name]
        out.append("")
        out.append(f"constexpr int k{name.title().replace('_', '')} = {len(terms)};")
        out.append(f"static const CioTerm k{name.title().replace('_', '')}Tab[{len(terms)}] = {{")
        for n, a in terms:
            out.append("    {{%s}, %s}," % (", ".join(map(str, n)), ", ".join(hexf(v) for v in a)))
        out.append("};")
    out.append("")
    out.append("}}  // namespace bqp::iau")
    return "\n".join(out) + "\n"


def main():
    root = Path(sys.argv[1] if len(sys.argv) > 1 else os.environ["BQP_REFERENCE_ROOT"])
    ls, pl, s06 = parse((root / TABLES).read_text())
    for n, _ in ls + pl:
        assert all(-128 <= v <= 127 for v in n)
    for terms in s06.values():
        for n, _ in terms:
            assert all(-128 <= v <= 127 for v in n)
    dst = Path(__file__).resolve().parent / "iau2000a_tables.h"
    dst.write_text(emit(ls, pl, s06))
    print(dst)


if __name__ == "__main__":
    main()
