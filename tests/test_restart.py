"""Checkpoint files in the reference's formats, pinned byte for byte.

The reference's CALF-20 example ships branch01/REVIVE and branch01/REVCON, written by its
`revive` (utility_pack.f:1772-1817) for the 90-CO2 state.  tests/golden/make_golden.py records
that state (guest coordinates, production flag, chainstats, energy) and the SHA-256 of both
files; writing the same state here must reproduce both files exactly, and reading our REVIVE
back (revread, utility_pack.f:1840-1878) must return the state."""
import hashlib
import json
import os

import numpy as np

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
