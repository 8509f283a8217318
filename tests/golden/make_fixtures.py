"""Regenerate the golden fixtures under tests/golden/ from the reference tree.

Run once in a container that has the reference checkout mounted:

    python tests/golden/make_fixtures.py [REFERENCE_ROOT]

It reads the reference's own recorded known-answer data -- nothing is
recomputed here -- and writes small JSON/text fixtures that travel with the
repository (the reference tree is not available where the GPU tests run):

* ``dir_r6_d15.txt``: the GOCE DIR-R6 gravity field truncated to degree/order
  15, the field the reference's Python binding embeds
  (``two_phase_transfer_rs/data/spher_const/GO_CONS_GCF_2_DIR_R6_d15.txt``).
  The same file is copied to ``bqp_b200/data/`` as the package's default field.
* ``orekit_gravity_dir_r6_d5.json``: the Orekit 13.1.2 d/o 5 gravity comparator
  (``lightyear_odeint_rs/tests/data/orekit_dir_r6_5x5_v1.json``): 5 positions,
  full / point-mass / non-central accelerations, abs 5e-11 m/s^2 + rel 2e-12.
* ``orekit_jb2008.json``: the Orekit JB2008 adapter fixture
  (``lightyear_odeint_rs/tests/data/orekit_jb2008_eci_adapter_v1.json``, 15
  cases: primitive JB2008 inputs -> density, body position -> geodetic
  altitude) plus the Orekit JAR literals pinned in ``jb_rs/src/jb2008.rs``
  (``orekit_local_input`` and the 91 ... 35000 km vectors, rel 5e-13).
* ``julier7_offsets.json``: the reference's literal sigma-point offsets of the
  7-point Julier simplex (``dust_ukf_rs/src/lib.rs``, JULIER_WHITENED_OFFSETS),
  as bit patterns.
* ``ref_tableaus.json``: every ``c``, ``a``, ``b``, ``e`` and ``e3`` entry of
  the reference's DOPRI5, DOP853 (12 active stages), Vern7 and Vern9 tables
  (``lightyear_odeint_rs/src/odesolve/tableau/*.rs``) as binary64 hex strings,
  evaluated as Rust evaluates its constant expressions (``rust_tableaus.py``).

The reference root is the first argument or the ``BQP_REFERENCE_ROOT``
environment variable.
"""
import json
import os
import re
import struct
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent


# Licence attribution carried in the field file itself ('#' lines are
# comments to the coefficient loaders).
ATTRIBUTION = """\
# GOCE DIR Release 6 gravity field (GO_CONS_EGM_GOC_2__20091009T000000_20131020T235959_0201),
# truncated to degree and order 15; the truncation is the only change.
# Source: ICGEM, https://icgem.gfz.de/ , DOI 10.5880/ICGEM.2019.004.
# Licence: Creative Commons Attribution 4.0 International (CC BY 4.0),
# https://creativecommons.org/licenses/by/4.0/
# Columns: degree, order, normalised C, normalised S.
"""


def hex_to_f64(h: str) -> float:
    return struct.unpack(">d", bytes.fromhex(h[2:]))[0]


def main(ref_root: str | None = None) -> None:
    ref_root = ref_root or os.environ.get("BQP_REFERENCE_ROOT")
    if not ref_root:
        raise SystemExit("usage: make_fixtures.py REFERENCE_ROOT (or set BQP_REFERENCE_ROOT)")
    ref = Path(ref_root) / "dust_transfer"
    crates = ref / "crates"

    # 1. DIR-R6 d/o 15 field
    src = crates / "two_phase_transfer_rs/data/spher_const/GO_CONS_GCF_2_DIR_R6_d15.txt"
    text = ATTRIBUTION + src.read_text()
    (HERE / "dir_r6_d15.txt").write_text(text)
    (REPO / "bqp_b200/data").mkdir(parents=True, exist_ok=True)
    (REPO / "bqp_b200/data/dir_r6_d15.txt").write_text(text)

    # 2. Orekit gravity comparator
    g = json.loads((crates / "lightyear_odeint_rs/tests/data/orekit_dir_r6_5x5_v1.json").read_text())
    grav = {
        "source": "lightyear_odeint_rs/tests/data/orekit_dir_r6_5x5_v1.json",
        "authority": g["authority"],
        "degree": 5,
        "gm_m3_s2": g["model"]["gm_m3_s2"],
        "reference_radius_m": g["model"]["reference_radius_m"],
        "absolute_tolerance_m_s2": g["evaluation"]["absolute_tolerance_m_s2"],
        "relative_tolerance": g["evaluation"]["relative_tolerance"],
        "cases": [
            {k: c[k] for k in ("name", "position_m", "full_m_s2", "point_mass_m_s2",
                                "orekit_noncentral_m_s2")}
            for c in g["cases"]
        ],
    }
    (HERE / "orekit_gravity_dir_r6_d5.json").write_text(json.dumps(grav, indent=1) + "\n")

    # 3. Orekit JB2008 fixture + JAR literals
    j = json.loads((crates / "lightyear_odeint_rs/tests/data/orekit_jb2008_eci_adapter_v1.json").read_text())
    cases = []
    for c in j["cases"]:
        e = c["expected"]
        cases.append({
            "id": c["id"],
            "jb_primitive_inputs": e["jb_primitive_inputs"],
            "density_kg_m3": e["density_kg_m3"],
            "satellite_body_m": e["satellite_body_m"],
            "satellite_geodetic": e["satellite_geodetic"],
        })
    src_jb = (crates / "jb_rs/src/jb2008.rs").read_text()
    m = re.search(r"fn orekit_local_input\(altitude_km: f64\) -> Jb2008Input \{(.*?)\n    \}\n", src_jb, re.S)
    body = m.group(1)

    def field(name):
        mm = re.search(name + r": ([^,\n]+),", body)
        return mm.group(1).strip()

    def num(s):
        return float(s.replace("_", ""))

    ha = field("hour_angle_rad")
    a, b = [num(x) for x in ha.split(" - ")]
    local = {
        "mjd_utc": num(field("mjd_utc")),
        "sun_declination_rad": num(field("sun_declination_rad")),
        "hour_angle_rad": a - b,
        "sat_geocentric_lat_rad": num(field("sat_geocentric_lat_rad")),
        "f10": num(field("f10")), "f10b": num(field("f10b")),
        "s10": num(field("s10")), "s10b": num(field("s10b")),
        "m10": num(field("m10")), "m10b": num(field("m10b")),
        "y10": num(field("y10")), "y10b": num(field("y10b")),
        "dtc_k": num(field("dst_temperature_correction_k")),
    }
    lits = []
    mm = re.search(r"fn matches_orekit_piecewise_boundary_vectors\(\) \{(.*?)\n    \}\n", src_jb, re.S)
    for alt, val in re.findall(r"\(([0-9.]+), ([0-9._e-]+)\)", mm.group(1)):
        lits.append({"altitude_km": num(alt), "mjd_utc": None, "density_kg_m3": num(val)})
    m400 = re.search(r"mjd_utc: ([0-9_.]+),\s*\.\.orekit_local_input\(([0-9.]+)\)\s*\}\)\s*\.unwrap\(\);\s*let expected = ([0-9._e-]+);", mm.group(1), re.S)
    lits.append({"altitude_km": num(m400.group(2)), "mjd_utc": num(m400.group(1)),
                 "density_kg_m3": num(m400.group(3))})
    for fn in ("matches_exact_orekit_jar_91km_vector", "matches_exact_orekit_jar_35000km_vector"):
        mm = re.search(r"fn " + fn + r"\(\) \{(.*?)\n    \}\n", src_jb, re.S)
        alt = re.search(r"orekit_local_input\(([0-9_.]+)\)", mm.group(1)).group(1)
        bits = re.search(r"f64::from_bits\((0x[0-9a-f_]+)\)", mm.group(1)).group(1).replace("_", "")
        lits.append({"altitude_km": num(alt), "mjd_utc": None, "density_kg_m3": hex_to_f64(bits)})
    # the coarse-profile (atm_model 5) receipts beside the exact ones, as bit
    # patterns (jb_rs/tests/jb2008_logquad_x4_probe.rs, shared-core checksum)
    probe = (crates / "jb_rs/tests/jb2008_logquad_x4_probe.rs").read_text()
    mm = re.search(r"fn shared_core_checksum_tracks_corrected_species_reduction_bits\(\) \{(.*?)\n\}\n", probe, re.S)
    x4 = []
    for alt, exact_bits, probe_bits in re.findall(r"\(([0-9_.]+), (0x[0-9a-f_]+), (0x[0-9a-f_]+)\)", mm.group(1)):
        x4.append({"altitude_km": num(alt), "exact": hex_to_f64("0x" + exact_bits[2:].replace("_", "")),
                   "model5": hex_to_f64("0x" + probe_bits[2:].replace("_", ""))})
    jb = {
        "source": ["lightyear_odeint_rs/tests/data/orekit_jb2008_eci_adapter_v1.json",
                   "jb_rs/src/jb2008.rs (orekit_local_input and Orekit JAR literal tests)",
                   "jb_rs/tests/jb2008_logquad_x4_probe.rs (exact and model-5 receipts)"],
        "model5_receipts": x4,
        "earth": j["earth"],
        "relative_tolerance": 5e-13,
        "cases": cases,
        "orekit_local_input": local,
        "literals": lits,
    }
    (HERE / "orekit_jb2008.json").write_text(json.dumps(jb, indent=1) + "\n")

    # 4. The reference's literal Julier simplex offsets (bit patterns)
    ukf = (crates / "dust_ukf_rs/src/lib.rs").read_text()
    body = re.search(r"static JULIER_WHITENED_OFFSETS: \[\[f64; DIM\]; NUM_SIGMA\] = \[(.*?)\n\];", ukf,
                     re.S).group(1)
    rows = []
    for row in re.findall(r"\[(.*?)\]", body, re.S):
        vals = []
        for tok in [t.strip() for t in row.split(",") if t.strip()]:
            m = re.match(r"f64::from_bits\((0x[0-9a-f_]+)\)", tok)
            vals.append(hex_to_f64("0x" + m.group(1)[2:].replace("_", "")) if m else float(tok))
        rows.append(vals)
    offs = {"source": "dust_ukf_rs/src/lib.rs (JULIER_WHITENED_OFFSETS)",
            "offsets": rows, "bits": [[struct.pack(">d", v).hex() for v in r] for r in rows]}
    (HERE / "julier7_offsets.json").write_text(json.dumps(offs, indent=1) + "\n")

    # 5. The reference's Runge-Kutta tables, bit for bit
    sys.path.insert(0, str(HERE))
    import rust_tableaus

    tabs = rust_tableaus.read_all(ref_root)

    def hx(v):
        return None if v is None else [float(x).hex() for x in v]

    tab_out = {"source": rust_tableaus.TABLEAU_DIR + "/{dopri5,dop853,dop853_coeffs,vern7,vern9}.rs",
               "tables": {name: {"stages": len(t["c"]), "c": hx(t["c"]), "a": [hx(r) for r in t["a"]],
                                 "b": hx(t["b"]), "e": hx(t["e"]), "e3": hx(t["e3"])}
                          for name, t in tabs.items()}}
    (HERE / "ref_tableaus.json").write_text(json.dumps(tab_out, indent=1) + "\n")
    print("fixtures written:", len(grav["cases"]), "gravity,", len(cases), "jb2008 cases,",
          len(lits), "jb2008 literals,", len(rows), "sigma offset rows,", len(tabs), "RK tables")


if __name__ == "__main__":
    main(*sys.argv[1:])
