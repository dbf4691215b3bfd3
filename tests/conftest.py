import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "fastmc-1.4.0_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs through the CUDA library)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle

    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def fmc():
    lib = os.path.join(PKG, "lib", "libfastmc_b200.so")
    if not os.path.exists(lib):
        subprocess.run([sys.executable, os.path.join(PKG, "build.py")], check=True)
    import fastmc_b200

    return fastmc_b200


@pytest.fixture(scope="session")
def decks(tmp_path_factory):
    """Synthetic input decks shared by the tests."""
    from fastmc_b200 import synth

    root = tmp_path_factory.mktemp("decks")
    out = {
        "small": synth.write_plain_small(str(root / "small")),
        "large": synth.write_plain_large(str(root / "large")),
        "calf20": os.path.join(GOLDEN, "calf20"),
    }
    fws = synth.batched_frameworks(3, seed=11)
    for i, fw in enumerate(fws):
        L = [fw.cell[j, j] for j in range(3)]
        out[f"ortho{i}"] = synth.write_inputs(str(root / f"ortho{i}"), fw, ["CO2"], [1.0], 298.0,
                                              tuple(synth.kmax_for(x) for x in L))
    L = [fws[1].cell[j, j] for j in range(3)]
    out["forms"] = synth.write_inputs(str(root / "forms"), fws[1], ["CO2"], [1.0], 298.0,
                                      tuple(synth.kmax_for(x) for x in L), vdw_forms=synth.VDW_FORMS)
    L = [fws[2].cell[j, j] for j in range(3)]
    out["jumps"] = synth.write_inputs(str(root / "jumps"), fws[2], ["CO2"], [1.0], 298.0,
                                      tuple(synth.kmax_for(x) for x in L),
                                      moves={"insert": 0.3, "delete": 0.25, "displace": 0.15, "jump": 0.15,
                                             "flex": 0.05, "swap": 0.05, "rotate": 0.05})
    # hot and dense enough that some multi-jumps are accepted: most random jumps overlap
    # framework atoms by tens of kcal/mol
    out["multijump"] = synth.write_inputs(str(root / "multijump"), fws[2], ["CO2"], [50000.0], 30000.0,
                                          tuple(synth.kmax_for(x) for x in L),
                                          moves={"insert": 0.3, "delete": 0.2, "multi": 0.3, "jump": 0.1,
                                                 "displace": 0.1})
    # the reference's restart example 2: a binary CO2 + TIP4P-Ew deck on the unary run's REVCON,
    # with the CO2 count set to the REVCON's 90 molecules as its README instructs
    binary = root / "binary_preloaded"
    shutil.copytree(os.path.join(GOLDEN, "binary_preloaded"), binary)
    fld = (binary / "FIELD").read_text().split("\n")
    fld[next(i for i, ln in enumerate(fld) if ln.startswith("NUMMOLS"))] = "NUMMOLS 90"
    (binary / "FIELD").write_text("\n".join(fld))
    out["binary_preloaded"] = str(binary)
    out["calf20_co2_n2"] = os.path.join(GOLDEN, "calf20_co2_n2")
    # the reference's single-gas examples: CO2 in CALF-20's primitive cell, N2 in MOMJIJ, CH4 in
    # MASMIC (all triclinic, 4 A cutoff)
    for name in ("simple_calf20_co2", "simple_momjij_n2", "simple_masmic_ch4"):
        out[name] = os.path.join(GOLDEN, name)
    out["guest_moves"] = os.path.join(GOLDEN, "guest_moves")
    # CO2 + N2 with the reference's pressure equilibration: the partial pressures move every 400
    # moves until the forced stop at 50 x 100 cycles, then equilibration and production follow
    peq = synth.write_inputs(str(root / "pressure_eq"), fws[0], ["CO2", "N2"], [0.5, 0.5], 298.0,
                             tuple(synth.kmax_for(fws[0].cell[j, j]) for j in range(3)), eq_cycles=-100,
                             prod_cycles=-5)
    ctl = open(os.path.join(peq, "CONTROL")).read().replace(
        "finish", "desorb 1\nadsorb press 0.3 0.7\nadsorb guests 6.0 2.0\npacking fraction 0.5\n"
                  "finishment 1e-9\nfinish")
    open(os.path.join(peq, "CONTROL"), "w").write(ctl)
    out["pressure_eq"] = peq
    # the half-shift cells: truncated octahedron, rhombic dodecahedron, hexagonal prism
    for imcon, edge in ((4, 30.0), (5, 26.0), (7, 26.0)):
        hf = synth.half_shift_framework(imcon, edge, seed=40 + imcon)
        out[f"imcon{imcon}"] = synth.write_inputs(str(root / f"imcon{imcon}"), hf, ["CO2"], [2.0], 298.0,
                                                  tuple(synth.kmax_for(hf.cell[j, j]) for j in range(3)),
                                                  imcon=imcon)
    slab = synth.slab_framework(26.0, 20.0, 60.0, seed=46)
    out["imcon6"] = synth.write_inputs(str(root / "imcon6"), slab, ["CO2"], [2.0], 298.0,
                                       tuple(synth.kmax_for(slab.cell[j, j]) for j in range(3)), imcon=6)
    fw = fws[0]
    out["mixture"] = synth.write_inputs(str(root / "mixture"), fw, ["CO2", "N2"], [0.15, 0.85], 298.0,
                                        tuple(synth.kmax_for(fw.cell[j, j]) for j in range(3)))
    return out
