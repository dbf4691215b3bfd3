"""Chains created from arrays (fmc_chain_create) and the split-array trial calls on the device.

* A deck read into a descriptor and created from it runs the identical trajectory, bit for bit,
  to the chain opened from the deck.
* Guests handed over in the descriptor (the unary CALF-20 REVIVE state) give the reference's
  stored energy, as the deck route with fmc_set_guests does.
* A descriptor built from the generator's own arrays (no files) gives the deck chain's single
  point, S(k) and trial-pass energies within 1e-9 relative (the two routes differ only by the
  printed precision of the deck).
* fmc_ewald1_guest_xyz / fmc_guest_realspace_xyz / fmc_commit_xyz equal the interleaved calls."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from desc_util import desc_from_synth
from test_gpu_plain import _random_guest

pytestmark = pytest.mark.gpu
REL = 1e-9


@pytest.mark.parametrize("deck", ["small", "mixture", "forms"])
def test_descriptor_chain_runs_the_deck_trajectory_bit_for_bit(fmc, decks, deck):
    seed = (27, 18, 28, 18)
    a = fmc.Chain(decks[deck], seed=seed)
    desc = fmc.SystemDesc.from_deck(decks[deck])
    b = fmc.Chain(desc, seed=seed)
    desc.free()  # the chain keeps nothing of the caller's arrays
    ta, tb = a.run(3000), b.run(3000)
    assert ta.tobytes() == tb.tobytes()
    assert np.array_equal(a.sk(), b.sk())


def test_descriptor_hands_over_preloaded_guests(fmc):
    calf = os.path.join(GOLDEN, "calf20")
    exp = json.load(open(os.path.join(calf, "expected.json")))
    guests = np.load(os.path.join(calf, "revive_guests.npy"))
    desc = fmc.SystemDesc.from_deck(calf)
    desc.set_guests(0, guests)
    b = fmc.Chain(desc, seed=exp["seed"])
    sp_b, dlp_b = b.single_point()
    assert abs(sp_b - exp["revive_energy_kcal"]) <= REL * abs(exp["revive_energy_kcal"])
    a = fmc.Chain(calf, seed=exp["seed"])
    a.set_guests(0, guests)
    sp_a, dlp_a = a.single_point()
    assert sp_a == sp_b and dlp_a == dlp_b
    assert np.array_equal(a.sk(), b.sk())


def test_descriptor_from_generator_arrays_matches_the_deck_chain(fmc, oracle_mod, decks):
    from fastmc_b200 import synth

    fw = synth.plain_small_framework()
    b = fmc.Chain(desc_from_synth(fmc, fw, synth.CO2, 0.15, 298.0, (8, 8, 8)), seed=(1, 2, 3, 4))
    a = fmc.Chain(decks["small"], seed=(1, 2, 3, 4))
    ia, ib = a.info(), b.info()
    assert ia["K"] == ib["K"]
    assert abs(ia["dlpeng"] - ib["dlpeng"]) <= REL * abs(ia["dlpeng"])
    sa, sb = a.sk(), b.sk()
    assert np.max(np.abs(sa - sb)) <= REL * np.max(np.abs(sa))
    tmpl, _, _, _ = oracle_mod.Chain(decks["small"]).guest_template(0)
    cell = fw.cell
    rng = np.random.default_rng(3)
    for _ in range(8):
        xyz = _random_guest(rng, tmpl, cell)
        ea, eb = a.ewald1_guest(0, xyz, fmc.INSERT), b.ewald1_guest(0, xyz, fmc.INSERT)
        assert abs(ea - eb) <= REL * abs(ea)
        (ra, va), (rb, vb) = a.guest_realspace(0, xyz), b.guest_realspace(0, xyz)
        scale = max(abs(ra), abs(va), 1.0)
        assert abs(ra - rb) <= REL * scale and abs(va - vb) <= REL * scale


def test_split_coordinate_calls_equal_the_interleaved_ones(fmc, oracle_mod, decks):
    d = decks["small"]
    a = fmc.Chain(d, seed=(5, 5, 5, 5))
    b = fmc.Chain(d, seed=(5, 5, 5, 5))
    a.run(300, trace=False)
    b.run(300, trace=False)
    tmpl, _, _, _ = oracle_mod.Chain(d).guest_template(0)
    lines = open(os.path.join(d, "CONFIG")).read().split("\n")
    cell = np.array([[float(v) for v in lines[k].split()] for k in (2, 3, 4)])
    rng = np.random.default_rng(8)
    xyz = _random_guest(rng, tmpl, cell)
    assert a.ewald1_guest(0, xyz, fmc.INSERT) == b.ewald1_guest_xyz(0, xyz[:, 0], xyz[:, 1], xyz[:, 2], fmc.INSERT)
    assert a.guest_realspace(0, xyz) == b.guest_realspace_xyz(0, xyz[:, 0], xyz[:, 1], xyz[:, 2])
    a.commit(fmc.INSERT, 0, -1, xyz)
    b.commit_xyz(fmc.INSERT, 0, -1, xyz[:, 0], xyz[:, 1], xyz[:, 2])
    assert np.array_equal(a.sk(), b.sk()) and np.array_equal(a.guest_coords(0), b.guest_coords(0))
    # a displacement (pass 1 old sites, pass 2 new) and its commit, then a deletion
    old = a.guest_coords(0)[0]
    new = old + np.array([0.2, 0.1, -0.3])
    a.ewald1_guest(0, old, fmc.DISPLACE, 1)
    b.ewald1_guest_xyz(0, old[:, 0], old[:, 1], old[:, 2], fmc.DISPLACE, 1)
    assert a.ewald1_guest(0, new, fmc.DISPLACE, 2) == b.ewald1_guest_xyz(0, new[:, 0], new[:, 1], new[:, 2],
                                                                         fmc.DISPLACE, 2)
    assert a.guest_realspace(0, new, 0) == b.guest_realspace_xyz(0, new[:, 0], new[:, 1], new[:, 2], 0)
    a.commit(fmc.DISPLACE, 0, 0, new)
    b.commit_xyz(fmc.DISPLACE, 0, 0, new[:, 0], new[:, 1], new[:, 2])
    assert a.ewald1_guest(0, new, fmc.DELETE) == b.ewald1_guest_xyz(0, new[:, 0], new[:, 1], new[:, 2], fmc.DELETE)
    a.commit(fmc.DELETE, 0, 0)
    b.commit_xyz(fmc.DELETE, 0, 0)
    assert np.array_equal(a.sk(), b.sk()) and np.array_equal(a.guest_coords(0), b.guest_coords(0))
