"""Checkpoint files in the reference's formats, pinned byte for byte.

The reference's CALF-20 example ships branch01/REVIVE and branch01/REVCON, written by its
`revive` (utility_pack.f:1772-1817) for the 90-CO2 state.  tests/golden/make_golden.py records
that state (guest coordinates, production flag, chainstats, energy) and the SHA-256 of both
files; writing the same state here must reproduce both files exactly, and reading our REVIVE
back (revread, utility_pack.f:1840-1878) must return the state."""
import hashlib
import json
import os
import shutil

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CALF = os.path.join(HERE, "golden", "calf20")


def _fixture():
    exp = json.load(open(os.path.join(CALF, "expected.json")))
    guests = np.load(os.path.join(CALF, "revive_guests.npy"))
    return exp, guests


def test_revive_and_revcon_match_the_reference_files(fmc, tmp_path):
    exp, guests = _fixture()
    fmc.write_revive_state(CALF, str(tmp_path), [guests], production=exp["revive_production"] != 0,
                           chainstats=exp["revive_chainstats"], energy=[exp["revive_energy_kcal"]], eng=0.0)
    for name, key in (("REVIVE", "revive_sha256"), ("REVCON", "revcon_sha256")):
        digest = hashlib.sha256(open(tmp_path / name, "rb").read()).hexdigest()
        assert digest == exp[key], name


def test_revive_round_trip(fmc, tmp_path):
    exp, guests = _fixture()
    fmc.write_revive_state(CALF, str(tmp_path), [guests], production=True, chainstats=exp["revive_chainstats"],
                           energy=[exp["revive_energy_kcal"]])
    r = fmc.read_revive(str(tmp_path / "REVIVE"), CALF)
    assert r["production"] is True
    assert r["natms"] == exp["revive_natms"]
    assert np.array_equal(r["guests"][0], guests)
    assert np.array_equal(r["chainstats"], np.asarray(exp["revive_chainstats"]))
    assert r["energy"][0] == exp["revive_energy_kcal"]


def test_revive_of_another_deck_is_rejected(fmc, tmp_path, decks):
    exp, guests = _fixture()
    fmc.write_revive_state(CALF, str(tmp_path), [guests], energy=[0.0])
    try:
        fmc.read_revive(str(tmp_path / "REVIVE"), decks["small"])
    except fmc.FastMCError as e:
        assert "REVIVE does not match" in str(e)
    else:
        raise AssertionError("a REVIVE of another FIELD was accepted")


@pytest.mark.parametrize("name", ["calf20_co2_n2", "simple_momjij_n2", "simple_masmic_ch4"])
def test_checkpoint_round_trip_on_the_shipped_decks(fmc, oracle_mod, decks, tmp_path, name):
    """REVIVE written for the reference's other example decks (two species; N2 with its massless
    centre site; single-site CH4) reads back as written, and REVCON used as the CONFIG of a new
    run with the FIELD's NUMMOLS set to the guest counts (the reference's own recipe for starting
    from a finished run, examples/restart/2 README) gives the oracle the same guests to the 10
    significant digits REVCON keeps, and the product the same k-vector tables."""
    d = decks[name]
    orc = oracle_mod.Chain(d)
    ng = fmc.deck_inspect(d)["nspecies"]
    assert ng == (2 if name == "calf20_co2_n2" else 1)
    rng = np.random.default_rng(17)
    guests, counts = [], []
    for g in range(ng):
        tmpl = orc.guest_template(g)[0]
        n = int(rng.integers(3, 9))
        com = rng.uniform(0.5, 8.0, (n, 1, 3))
        guests.append(com + tmpl[None, :, :])
        counts.append(n)
    cs = rng.normal(size=1 + 14 * ng)
    en = rng.normal(size=ng)
    fmc.write_revive_state(d, str(tmp_path), guests, production=True, chainstats=cs, energy=en, eng=-1.25)
    r = fmc.read_revive(str(tmp_path / "REVIVE"), d)
    assert r["production"] is True
    for g in range(ng):
        assert np.array_equal(r["guests"][g], guests[g])
    assert np.array_equal(r["chainstats"], cs) and np.array_equal(r["energy"], en)
    # REVCON as the next run's CONFIG
    nxt = tmp_path / "next"
    os.makedirs(nxt)
    for f in ("CONTROL",):
        shutil.copy(os.path.join(d, f), nxt / f)
    field = open(os.path.join(d, "FIELD")).read().split("\n")
    k = 0
    for i, line in enumerate(field):
        if line.strip().upper() == "NUMMOLS 0" and k < ng:
            field[i] = "NUMMOLS %d" % counts[k]
            k += 1
    assert k == ng
    (nxt / "FIELD").write_text("\n".join(field))
    shutil.copy(tmp_path / "REVCON", nxt / "CONFIG")
    xyz, _, _, _ = oracle_mod.Chain(str(nxt)).atoms()
    want = np.concatenate([g.reshape(-1, 3) for g in guests])
    assert np.allclose(xyz[: len(want)], want, rtol=0, atol=1e-8)
    a, b = fmc.deck_inspect(str(nxt)), fmc.deck_inspect(d)
    assert np.array_equal(a["lmn"], b["lmn"]) and np.array_equal(a["akk"], b["akk"])
    assert a["nframework"] == b["nframework"]
