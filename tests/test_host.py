"""Host logic of the product (no GPU): C-ABI exports, deck reading and tables against the oracle,
the reference's error codes."""
import os
import re
import shutil

import numpy as np
import pytest

from conftest import ROOT


def header_symbols():
    text = open(os.path.join(ROOT, "include", "fastmc_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fmc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(fmc):
    import ctypes

    from fastmc_b200 import _lib

    L = ctypes.CDLL(_lib.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_lib.SIGNATURES), "python binding and header disagree"
    assert L.fmc_version() == 10400


@pytest.mark.parametrize("name", ["calf20", "small", "large", "ortho0", "ortho1", "mixture", "imcon4", "imcon5",
                                  "imcon6", "imcon7", "simple_calf20_co2", "simple_momjij_n2",
                                  "simple_masmic_ch4"])
def test_deck_tables_match_oracle_bit_exact(fmc, oracle_mod, decks, name):
    info = fmc.deck_inspect(decks[name])
    orc = oracle_mod.Chain(decks[name])
    lmn, akk = orc.kvectors()
    assert info["K"] == len(akk)
    assert np.array_equal(info["lmn"], lmn)
    assert np.array_equal(info["akk"], akk)
    assert np.array_equal(info["erc"], orc.erc())
    s = orc.scalars()
    for k in ("alpha", "rcut", "volm", "engunit", "beta", "drewd", "dlrpot", "statvolm"):
        assert info[k] == s[k], k
    _, q, _, _ = orc.atoms()
    assert np.array_equal(info["charges"], q[len(q) - info["nframework"]:])


def test_every_vdw_form_tabulates_like_the_oracle(fmc, oracle_mod, decks):
    """The nine pair forms of forgen (vdw_terms.f:190-396), each used by some pair of the deck."""
    field = open(decks["forms"] + "/FIELD").read().lower()
    for form in ("12-6", " lj ", " nm ", "buck", " bhm ", "hbnd", " snm ", "mors", " wca "):
        assert form in field, form
    tabs = fmc.deck_vdw(decks["forms"])
    orc = oracle_mod.Chain(decks["forms"])
    ntpvdw = int(next(l for l in field.splitlines() if l.startswith("vdw")).split()[1])
    assert ntpvdw >= 9 and len(tabs) >= ntpvdw
    for k in range(1, ntpvdw + 1):
        assert np.array_equal(tabs[k - 1], orc.vvv(k)), k


@pytest.mark.parametrize("name", ["calf20", "simple_momjij_n2", "simple_masmic_ch4", "calf20_co2_n2"])
def test_shipped_example_vdw_tables_match_the_oracle(fmc, oracle_mod, decks, name):
    """The vdW pair tables of the reference's own example decks (lj pairs of MOF atoms with the
    guests' sites, zero-table pairs where FIELD gives none)."""
    tabs = fmc.deck_vdw(decks[name])
    orc = oracle_mod.Chain(decks[name])
    field = open(decks[name] + "/FIELD").read().lower().splitlines()
    ntpvdw = int(next(l for l in field if l.startswith("vdw")).split()[1])
    assert ntpvdw > 0 and len(tabs) >= ntpvdw
    for k in range(1, ntpvdw + 1):
        assert np.array_equal(tabs[k - 1], orc.vvv(k)), k


def _copy_deck(src, dst):
    shutil.copytree(src, dst)
    return dst


def _edit(path, old, new):
    t = open(path).read()
    assert old in t
    open(path, "w").write(t.replace(old, new, 1))


CASES = [
    ("CONTROL", "temperature", "# temperature", 380),   # temperature missing
    ("CONTROL", "move insert", "wibble insert", 3),     # unknown directive
    ("CONTROL", "ewald sum", "# ewald sum", 2311),      # no Ewald sum
    ("CONTROL", "&guest 1", "&guest 2", 2312),          # guest index not in FIELD
    ("CONTROL", "finish", "", 53),                      # CONTROL ends early
    ("CONFIG", "Zn   ", "Qq   ", 25),                   # wrong atom label
    ("FIELD", "close", "", 52),                         # FIELD ends early
    ("FIELD", "UNITS kcal", "UNITS kcal\nbogus line", 4),  # unknown FIELD directive
    ("CONTROL", "cutoff 12.500000", "cutoff 14.000000", 95),  # cutoff beyond half width
]


@pytest.mark.parametrize("fname,old,new,code", CASES)
def test_reference_error_codes(fmc, oracle_mod, decks, tmp_path, fname, old, new, code):
    d = _copy_deck(decks["small"], str(tmp_path / "deck"))
    _edit(os.path.join(d, fname), old, new)
    with pytest.raises(fmc.FastMCError) as e:
        fmc.deck_inspect(d)
    assert e.value.code == code
    with pytest.raises(oracle_mod.OracleError) as eo:
        oracle_mod.Chain(d)
    assert eo.value.code == code


def test_cubic_cell_consistency_error_410(fmc, oracle_mod, decks, tmp_path):
    d = _copy_deck(decks["small"], str(tmp_path / "deck"))
    lines = open(os.path.join(d, "CONFIG")).read().split("\n")
    lines[3] = "".join(f"{v:20.12f}" for v in (0.0, 25.9, 0.0))
    open(os.path.join(d, "CONFIG"), "w").write("\n".join(lines))
    with pytest.raises(fmc.FastMCError) as e:
        fmc.deck_inspect(d)
    assert e.value.code == 410
    with pytest.raises(oracle_mod.OracleError) as eo:
        oracle_mod.Chain(d)
    assert eo.value.code == 410


def test_dblstr_semantics_through_ewald_line(fmc, oracle_mod, decks, tmp_path):
    # 'ewald precision 1d-6' goes through the DL_POLY precision rule in both readers
    d = _copy_deck(decks["small"], str(tmp_path / "deck"))
    _edit(os.path.join(d, "CONTROL"), "ewald sum 0.260000 8 8 8", "ewald precision 1d-6")
    info = fmc.deck_inspect(d)
    orc = oracle_mod.Chain(d)
    i = orc.ints()
    assert (info["kmax1"], info["kmax2"], info["kmax3"]) == (i["kmax1"], i["kmax2"], i["kmax3"])
    assert info["alpha"] == orc.scalars()["alpha"]
    assert info["K"] == i["newld"]


def test_host_voxel_lists_are_ascending_and_complete(fmc, decks):
    """fmc_deck_voxels (the host's every-atom test): CSR offsets, ascending atom indices per voxel,
    and every atom in the list of the voxel that holds it."""
    nvox, off, atoms = fmc.deck_voxels(decks["ortho0"], 2.0)
    info = fmc.deck_inspect(decks["ortho0"])
    assert off[0] == 0 and off[-1] == atoms.size and np.all(np.diff(off) >= 0)
    assert atoms.min() >= 0 and atoms.max() < info["nframework"]
    for v in range(0, int(np.prod(nvox)), 37):
        seg = atoms[off[v]:off[v + 1]]
        assert np.all(np.diff(seg) > 0)
    assert len(np.unique(atoms)) == info["nframework"]


def test_deck_reader_line_endings(fmc, decks, tmp_path):
    """The reader takes each file whole and splits it the way line-by-line reading does: CRLF
    line endings and a last line without a newline give the same deck, table for table."""
    src = decks["small"]
    dst = tmp_path / "crlf"
    dst.mkdir()
    for name in ("CONTROL", "FIELD", "CONFIG"):
        text = open(os.path.join(src, name)).read()
        crlf = text.replace("\n", "\r\n")
        if name == "CONFIG":
            crlf = crlf.rstrip("\r\n")  # no newline after the last record
        (dst / name).write_bytes(crlf.encode())
    a, b = fmc.deck_inspect(src), fmc.deck_inspect(str(dst))
    for k in ("K", "natoms", "nframework", "ntypes", "mxgrid", "nvoxels"):
        assert a[k] == b[k], k
    for k in ("alpha", "rcut", "volm", "temp", "beta"):
        assert a[k] == b[k], k
    for k in ("lmn", "akk", "erc", "charges"):
        assert np.array_equal(a[k], b[k]), k
    nv_a, off_a, at_a = fmc.deck_voxels(src, 2.0)
    nv_b, off_b, at_b = fmc.deck_voxels(str(dst), 2.0)
    assert nv_a == nv_b and np.array_equal(off_a, off_b) and np.array_equal(at_a, at_b)


def test_batch_tile_table(fmc):
    """The batched kernel's tile shapes (host only): tile 0 the default, every shape once, the
    thread counts the autotuner chooses among."""
    tiles = fmc.batch_tiles()
    assert tiles[0] == (256, 1, 1)
    assert len(set(tiles)) == len(tiles) == 12
    assert {t[0] for t in tiles} == {128, 256, 384}
    assert {t[1] for t in tiles} == {1, 2} and {t[2] for t in tiles} == {1, 2}


def test_deck_reader_matches_oracle_parser_on_random_decks(fmc, oracle_mod, tmp_path):
    """The library's deck reader (whole-file reads, correctly rounded coordinate parsing) against
    the oracle's own restatement of readinputs.f on request decks of random size, gas and
    conditions: framework coordinates, charges, k-vectors and erfc table bit for bit."""
    from fastmc_b200 import synth

    for r in synth.serving_requests(12, seed=23):
        r["natoms"] = min(r["natoms"], 1500)  # keep the oracle's set-up quick
        r["edge"] = max((r["natoms"] / 0.025) ** (1.0 / 3.0), 25.2)
        d = synth.write_request(str(tmp_path / f"r{r['id']}"), r)
        desc = fmc.SystemDesc.from_deck(d)
        nf = desc.s.nframework
        xyz = np.ctypeslib.as_array(desc.s.fw_xyz, shape=(3 * nf,)).reshape(nf, 3)
        q = np.ctypeslib.as_array(desc.s.fw_charge, shape=(nf,))
        orc = oracle_mod.Chain(d)
        oxyz, oq, _, _ = orc.atoms()
        assert np.array_equal(xyz, oxyz[len(oq) - nf:]), r["id"]
        assert np.array_equal(q, oq[len(oq) - nf:]), r["id"]
        info = fmc.deck_inspect(d)
        lmn, akk = orc.kvectors()
        assert np.array_equal(info["lmn"], lmn) and np.array_equal(info["akk"], akk)
        assert np.array_equal(info["erc"], orc.erc())
        s = orc.scalars()
        for k in ("temp", "alpha", "rcut", "volm", "beta", "statvolm"):
            assert info[k] == s[k], (r["id"], k)
