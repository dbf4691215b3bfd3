"""Regenerate the golden fixtures under tests/golden/ from the reference's shipped example.

Run in a container where the reference checkout is mounted (default /root/reference):

    python tests/golden/make_golden.py [/path/to/reference]

It copies the CALF-20 example inputs (CONTROL, FIELD, CONFIG) of
examples/restart/1_restart_example_with_completed_long_simulation_data/ and converts the
final chain state in branch01/REVIVE (Fortran unformatted sequential records, layout of
revive, utility_pack.f:1800-1815) into revive_guests.npy.  The known answers recorded in
expected.json come from that example's OUTPUT and REVIVE:

* OUTPUT:108  duni seed "103 112 53 153"
* OUTPUT:113  "Energy reported by DL_POLY: -11190.606165" (empty framework, recip + self)
* REVIVE      energy(1) = -731.5072668178669 kcal/mol for the 90-CO2 state it stores
* examples/advance/1_probability_plot_unary inputs, and atmnumber's mass windows as data
* REVIVE      its production flag, chainstats and natms, and the SHA-256 of REVIVE and REVCON,
              so that a writer restating revive (utility_pack.f:1772-1817) can be checked
              byte for byte without the files themselves
* OUTPUT      the per-node report block (report_node0.txt), to check the report writer's layout
* examples/advance/2 and 3, examples/restart/2 and examples/simple/1-3 inputs as further parity
  decks
"""
import hashlib
import json
import os
import shutil
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
EXAMPLE = "examples/restart/1_restart_example_with_completed_long_simulation_data"


def read_fortran_records(path):
    data = open(path, "rb").read()
    recs, o = [], 0
    while o < len(data):
        n = struct.unpack("<i", data[o:o + 4])[0]
        recs.append(data[o + 4:o + 4 + n])
        tail = struct.unpack("<i", data[o + 4 + n:o + 8 + n])[0]
        assert tail == n, "corrupt record marker"
        o += 8 + n
    return recs


def main(ref):
    src = os.path.join(ref, EXAMPLE)
    out = os.path.join(HERE, "calf20")
    os.makedirs(out, exist_ok=True)
    for f in ("CONTROL", "FIELD", "CONFIG"):
        shutil.copyfile(os.path.join(src, f), os.path.join(out, f))
    recs = read_fortran_records(os.path.join(src, "branch01", "REVIVE"))
    nummols = np.frombuffer(recs[1], "<i4")
    nco2 = int(nummols[0])
    gx, gy, gz = (np.frombuffer(recs[4 + i], "<f8") for i in range(3))
    guests = np.stack([gx, gy, gz], axis=1).reshape(nco2, 3, 3)
    energy = float(np.frombuffer(recs[-1], "<f8")[0])
    production = int(np.frombuffer(recs[0], "<i4")[0])
    chainstats = [float(v) for v in np.frombuffer(recs[2], "<f8")]
    natms = int(np.frombuffer(recs[3], "<i4")[0])
    sha = {f: hashlib.sha256(open(os.path.join(src, "branch01", f), "rb").read()).hexdigest()
           for f in ("REVIVE", "REVCON")}
    np.save(os.path.join(out, "revive_guests.npy"), guests)
    expected = {
        "seed": [103, 112, 53, 153],
        "dlpeng_empty_kcal": -11190.606165,
        "dlpeng_empty_digits": 6,
        "kmax": [9, 8, 8],
        "K": 870,
        "revive_nummols": [int(v) for v in nummols],
        "revive_energy_kcal": energy,
        "revive_production": production,
        "revive_chainstats": chainstats,
        "revive_natms": natms,
        "revive_sha256": sha["REVIVE"],
        "revcon_sha256": sha["REVCON"],
        "source": EXAMPLE + " (OUTPUT lines 108, 113; branch01/REVIVE)",
    }
    with open(os.path.join(out, "expected.json"), "w") as f:
        json.dump(expected, f, indent=1)
    print("wrote", out)
    # the probability-plot example's inputs (two plots of CO2: site 1; sites 2 and 3)
    pp = os.path.join(HERE, "probplot")
    os.makedirs(pp, exist_ok=True)
    for f in ("CONTROL", "FIELD", "CONFIG"):
        shutil.copyfile(os.path.join(ref, "examples/advance/1_probability_plot_unary", f), os.path.join(pp, f))
    print("wrote", pp)
    # the mass windows of atmnumber (utility_pack.f:1992-2237) as data, to check the writer's
    # atomic numbers against them
    import re
    upack = open(os.path.join(ref, "fastmc", "utility_pack.f")).read()
    body = upack[upack.index("integer function atmnumber"):upack.index("end function atmnumber")]
    wins = [[float(lo), float(hi), int(z)] for lo, hi, z in
            re.findall(r"\(i\.ge\.([0-9.]+)\)\.and\.\(i\.le\.([0-9.]+)\)\)then\s*\n\s*atmnumber=(\d+)", body)]
    with open(os.path.join(HERE, "atmnumber_windows.json"), "w") as f:
        json.dump(wins, f)
    print("wrote", len(wins), "atmnumber windows")
    # the other shipped examples as parity decks: a CO2/N2 mixture with probability plots, guest-
    # specific move and acceptance directives, the three single-gas examples (CO2 in CALF-20's
    # primitive cell, N2 in MOMJIJ, CH4 in MASMIC) and a binary CO2 + TIP4P-Ew deck whose CONFIG
    # is the unary run's REVCON (its README's recipe; the test sets the CO2 NUMMOLS)
    for name, sub in (("calf20_co2_n2", "examples/advance/2_absorbtion_of_co2_n2_in_calf-20"),
                      ("guest_moves", "examples/advance/3_guest_specific_move"),
                      ("simple_calf20_co2", "examples/simple/1_absorbtion_of_co2_in_calf-20"),
                      ("simple_momjij_n2", "examples/simple/2_absorbtion_of_n2_in_MOMJIJ"),
                      ("simple_masmic_ch4", "examples/simple/3_absorbtion_of_ch4_in_MASMIC")):
        dst = os.path.join(HERE, name)
        os.makedirs(dst, exist_ok=True)
        for f in ("CONTROL", "FIELD", "CONFIG"):
            shutil.copyfile(os.path.join(ref, sub, f), os.path.join(dst, f))
        print("wrote", dst)
    ex2 = os.path.join(ref, "examples/restart/2_start_binary_from_pre-loaded_unary_outputs")
    dst = os.path.join(HERE, "binary_preloaded")
    os.makedirs(dst, exist_ok=True)
    for f in ("CONTROL", "FIELD"):
        shutil.copyfile(os.path.join(ex2, "binary_from_pre-loaded_configuration", f), os.path.join(dst, f))
    shutil.copyfile(os.path.join(ex2, "pre-loaded_configuration", "branch01", "REVCON"), os.path.join(dst, "CONFIG"))
    print("wrote", dst)
    # the per-node report block of the example's OUTPUT (gcmc.f:2052-2108): from the blank line
    # before the banner through the blank line after the species block
    lines = open(os.path.join(src, "OUTPUT")).read().split("\n")
    i0 = next(i for i, s in enumerate(lines) if "Data reported from node" in s) - 2
    i1 = next(i for i in range(i0, len(lines)) if "Heat capacity error" in lines[i]) + 1
    with open(os.path.join(out, "report_node0.txt"), "w") as f:
        f.write("\n".join(lines[i0:i1 + 1]) + "\n")
    print("wrote report block, OUTPUT lines", i0 + 1, "-", i1 + 1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
