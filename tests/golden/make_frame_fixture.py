"""Regenerate ``tests/golden/frame_time.json`` from the reference tree.

Run once in a container that has the reference checkout mounted:

    python tests/golden/make_frame_fixture.py [REFERENCE_ROOT]

It copies the reference's recorded known answers for its IAU 2006/2000A
frame chain -- nothing is recomputed here:

* ``erfa``: the ERFA v2.0.1 ``t_erfa_c.c`` unit-test values the reference's
  own gates use, with ERFA's tolerances: ``satpy_core/src/frame_time/
  iau2006.rs`` gate 3 (xys06a, nut00a, nut06a, obl06, pfw06), ``cio.rs``
  gate 4 (c2ixys, sp00, pom00) and ``era.rs`` gate 2 (era00).
* ``cases``: the 20 cases of ``satpy_core/tests/data/erfa_sofa_derived_
  frame_time_v1.json`` (five UTC epochs, zero and real EOP): R, Rdot and
  Rddot of GCRS->ITRS from the five-point stencil with h = 0.25 s, a GCRS
  position / velocity / acceleration and its ITRS image, and for
  the real-EOP cases the four ``finals2000A.all`` records (MJD centre-1 ..
  centre+2) the chain interpolates, read with the reference's column rules
  (``frame_time/eop.rs`` load_eop: MJD 7..15, x_p 18..27, y_p 37..46,
  UT1-UTC 58..68, dX 97..106, dY 116..125).
* ``authority``: for the epochs of the reference's segment-cache test
  (``authority.rs`` segment_cache_matches_the_exact_chain_within_the_
  declared_bound) ten consecutive records of the sealed ``eop_table.bin``
  (five little-endian binary64 per UTC day from MJD 41684) around each, and
  the same days from ``finals2000A.all``, as numbers and as the raw text
  lines (the input of the library's finals reader).

Bounds stay in the tests that read the file; binary64 values are stored as
hex strings.
"""
import json
import os
import re
import struct
import sys
from datetime import date
from pathlib import Path

FT = "dust_transfer/crates/satpy_core/src/frame_time"
FIXTURE = "dust_transfer/crates/satpy_core/tests/data/erfa_sofa_derived_frame_time_v1.json"
FINALS = "dust_transfer/assets/reference/frame_time/finals2000A.all"
SEALED_FIRST_MJD = 41684

EPOCHS = {
    "2000-01-01T12:00:00": (2000, 1, 1, 12, 0, 0.0),
    "2016-12-31T23:59:59": (2016, 12, 31, 23, 59, 59.0),
    "2016-12-31T23:59:60": (2016, 12, 31, 23, 59, 60.0),
    "2017-01-01T00:00:00": (2017, 1, 1, 0, 0, 0.0),
    "2024-01-01T00:00:00": (2024, 1, 1, 0, 0, 0.0),
}
AUTHORITY_EPOCHS = [(2022, 8, 12, 4, 25, 0.0), (2022, 8, 12, 4, 55, 30.0), (2024, 1, 1, 0, 0, 0.0),
                    (2017, 1, 1, 0, 0, 0.0)]


def h64(x):
    return "0x" + struct.pack(">d", float(x)).hex()


def mjd_of(y, m, d):
    return (date(y, m, d) - date(1858, 11, 17)).days


def bits_in(src, fn_name):
    """Hex bit patterns (f64::from_bits) of one test function, in order."""
    start = src.index(f"fn {fn_name}")
    end = src.find("\n    #[test]", start + 1)
    body = src[start:end if end > 0 else len(src)]
    return ["0x" + h.replace("_", "") for h in re.findall(r"from_bits\(0x([0-9a-f_]+)\)", body)]


def finals_lines(text):
    """Raw text line of each MJD that has one of 125 characters or more."""
    lines = {}
    for line in text.splitlines():
        if len(line) >= 125:
            lines[int(float(line[7:15]))] = line
    return lines


def finals_rows(text):
    rows = {}
    for line in text.splitlines():
        if len(line) < 125:
            continue
        mjd = int(float(line[7:15]))
        try:
            rows[mjd] = [float(line[a:b]) for a, b in ((18, 27), (37, 46), (58, 68), (97, 106), (116, 125))]
        except ValueError:  # predicted days without nutation offsets
            continue
    return rows


def main(ref_root=None):
    root = Path(ref_root or os.environ["BQP_REFERENCE_ROOT"])
    iau = bits_in((root / FT / "iau2006.rs").read_text(), "gate3_xys06a_and_nutation")
    cio = bits_in((root / FT / "cio.rs").read_text(), "gate4_cio_and_polar_motion")
    era = bits_in((root / FT / "era.rs").read_text(), "gate2_era00_canonical")
    assert len(iau) == 12 and len(cio) == 11 and len(era) == 1, (len(iau), len(cio), len(era))
    erfa = {
        "xys06a": {"date": [2400000.5, 53736.0], "want": iau[0:3], "tol": [1e-14, 1e-15, 1e-18]},
        "nut00a": {"date": [2400000.5, 53736.0], "want": iau[3:5], "tol": [1e-13, 1e-13]},
        "nut06a": {"date": [2400000.5, 53736.0], "want": iau[5:7], "tol": [1e-13, 1e-13]},
        "obl06": {"date": [2400000.5, 54388.0], "want": iau[7:8], "tol": [1e-14]},
        "pfw06": {"date": [2400000.5, 50123.9999], "want": iau[8:12], "tol": [1e-16, 1e-12, 1e-14, 1e-12]},
        # c2ixys(x, y, s): elements [0][0], [0][2], [1][1], [2][0] (= x), [2][2]
        "c2ixys": {"xys": cio[0:3], "want": cio[3:7], "elements": [0, 2, 4, 8], "x_element": 6, "tol": 1e-13},
        "sp00": {"date": [2400000.5, 52541.0], "want": cio[7:8], "tol": [1e-24]},
        # pom00(xp, yp, sp): elements [0][0], [0][2], [1][1]
        "pom00": {"args": [2.55060238e-7, 1.860359247e-6, -1.3671745807288915e-11], "want": cio[8:11],
                  "elements": [0, 2, 4], "tol": [1e-13, 1e-16, 1e-13]},
        "era00": {"date": [2400000.5, 54388.0], "want": era, "tol": [1e-12]},
    }

    fixture = json.loads((root / FIXTURE).read_text())
    finals = finals_rows((root / FINALS).read_text())
    raw = finals_lines((root / FINALS).read_text())
    cases = []
    for c in fixture["cases"]:
        y, m, d, hh, mi, ss = EPOCHS[c["epoch_utc"]]
        real = c["eop_policy"] == "real_eop"
        centre = mjd_of(y, m, d)
        cases.append({
            "id": c["id"], "epoch": [y, m, d, hh, mi, ss], "policy": 1 if real else 0,
            "eop_first_mjd": centre - 1 if real else 0,
            "eop": [[h64(v) for v in finals[k]] for k in range(centre - 1, centre + 3)] if real else [],
            "R": c["R_gcrs_to_itrs"], "Rdot": c["Rdot_s1"], "Rddot": c["Rddot_s2"],
            "r_gcrs": c["r_gcrs_km"], "v_gcrs": c["v_gcrs_km_s"], "a_gcrs": c["a_gcrs_km_s2"],
            "r_itrs": c["r_itrs_km"], "v_itrs": c["v_itrs_km_s"], "a_itrs": c["a_itrs_km_s2"],
        })
    assert len(cases) == 20

    sealed = (root / FT / "eop_table.bin").read_bytes()
    auth = []
    for (y, m, d, hh, mi, ss) in AUTHORITY_EPOCHS:
        first = mjd_of(y, m, d) - 4
        rec = []
        for k in range(first, first + 10):
            off = (k - SEALED_FIRST_MJD) * 40
            rec.append([h64(v) for v in struct.unpack("<5d", sealed[off:off + 40])])
        auth.append({"epoch": [y, m, d, hh, mi, ss], "first_mjd": first, "sealed": rec,
                     "finals": [[h64(v) for v in finals[k]] for k in range(first, first + 10)],
                     "finals_lines": [raw[k] for k in range(first, first + 10)]})

    out = {
        "source": "tdude78/bqp dust_transfer satpy_core frame_time (ERFA 2.0.1 / SOFA 20231011-derived)",
        "erfa": erfa,
        "stencil_h_s": 0.25,
        "cases": cases,
        "authority": auth,
    }
    dst = Path(__file__).resolve().parent / "frame_time.json"
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print(dst)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
