"""The FP64 oracle against every known answer the reference ships (no GPU needed)."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

CALF = os.path.join(GOLDEN, "calf20")


def expected():
    with open(os.path.join(CALF, "expected.json")) as f:
        return json.load(f)


def test_duni_matches_published_universal_generator_vector(oracle_mod):
    # Marsaglia-Zaman universal generator known answer (F. James, Comput. Phys. Commun. 60
    # (1990) 329, RANMAR test): seeds (12,34,56,78); numbers 20001..20006 times 4096^2.
    s = oracle_mod.duni_stream((12, 34, 56, 78), 20006)
    assert (s[20000:] * 4096.0 * 4096.0).tolist() == [6533892.0, 14220222.0, 7275067.0, 6172232.0, 8354498.0,
                                                       10633180.0]


def test_calf20_precision_rule_and_kvectors(oracle_mod):
    c = oracle_mod.Chain(CALF, seed=expected()["seed"])
    i = c.ints()
    assert [i["kmax1"], i["kmax2"], i["kmax3"]] == expected()["kmax"]
    assert i["newld"] == expected()["K"]
    assert i["imcon"] == 3
    assert abs(c.scalars()["alpha"] - 0.25396) < 5e-6


def test_calf20_empty_framework_energy_pin(oracle_mod):
    c = oracle_mod.Chain(CALF, seed=expected()["seed"])
    # printed with 6 decimals in the reference OUTPUT
    assert abs(c.scalars()["dlpeng"] - expected()["dlpeng_empty_kcal"]) <= 5e-7


def test_revive_state_single_point_pin(oracle_mod):
    c = oracle_mod.Chain(CALF, seed=expected()["seed"])
    guests = np.load(os.path.join(CALF, "revive_guests.npy"))
    c.load_guests(0, guests.reshape(-1, 3))
    e = c.scalars()["spenergy"]
    ref = expected()["revive_energy_kcal"]
    assert abs(e - ref) / abs(ref) < 1e-9


def test_move_loop_energy_bookkeeping(oracle_mod, decks):
    c = oracle_mod.Chain(decks["small"], seed=(12, 34, 56, 78))
    tr = c.run(3000)
    acc = tr["accepted"] == 1
    assert np.isclose(np.sum(tr["estep"][acc]), tr["energy_after"][-1], rtol=0, atol=1e-6)
    # every insert attempt while empty is forced; molecule count changes only on accepted ins/del
    dn = np.diff(np.concatenate([[0], tr["nmols_after"]]))
    assert np.all(dn[(tr["mtype"] == 1) & acc] == 1)
    assert np.all(dn[(tr["mtype"] == 2) & acc] == -1)
    assert np.all(dn[~acc] == 0)
    # the running energy equals a fresh single point of the final state (drift bound)
    coords = c.guest_coords(0)
    e_run = c.scalars()["energy"]
    c2 = oracle_mod.Chain(decks["small"], seed=(12, 34, 56, 78))
    c2.load_guests(0, coords.reshape(-1, 3))
    assert abs(c2.scalars()["spenergy"] - e_run) <= 1e-8 * max(1.0, abs(e_run))


def test_rng_draw_order_displacement_skips_rande_when_downhill(oracle_mod, decks):
    c = oracle_mod.Chain(decks["small"], seed=(12, 34, 56, 78))
    tr = c.run(3000)
    disp = np.isin(tr["mtype"], [3, 4, 5])
    down = disp & (tr["estep"] < 0)
    assert np.all(tr["rande"][down] == -1.0)
    assert np.all(tr["accepted"][down] == 1)


def test_multi_jump_commits_or_restores_both_molecules(oracle_mod, decks):
    """Multiple long jumps (gcmc.f:1557-1785): two distinct molecules jump, one acceptance test
    on the summed energy change; on rejection both molecules and S(k) return to where they
    were.  The running energy must stay equal to a fresh single point of the state."""
    c = oracle_mod.Chain(decks["multijump"], seed=(12, 34, 56, 78))
    tr = c.run(2500)
    mj = tr["mtype"] == 8
    acc = tr["accepted"] == 1
    assert mj.sum() > 500 and 0 < (mj & acc).sum() < mj.sum()
    e = np.concatenate([[0.0], tr["energy_after"]])
    de = np.diff(e)
    # a rejected multi-jump leaves the energy where it was; an accepted one adds the summed dE
    assert np.all(de[mj & ~acc] == 0.0)
    assert np.allclose(de[mj & acc], tr["estep"][mj & acc], rtol=1e-12, atol=1e-9)
    # the molecule count never changes on a multi-jump
    n = np.concatenate([[0], tr["nmols_after"]])
    assert np.all(np.diff(n)[mj] == 0)
    coords = c.guest_coords(0)
    e_run = c.scalars()["energy"]
    c2 = oracle_mod.Chain(decks["multijump"], seed=(12, 34, 56, 78))
    c2.load_guests(0, coords.reshape(-1, 3))
    assert abs(c2.scalars()["spenergy"] - e_run) <= 1e-8 * max(1.0, abs(e_run))


def test_binary_deck_on_unary_revcon_single_point_pin(oracle_mod, decks):
    """The reference's restart example 2 (a binary CO2 + TIP4P-Ew run started from the unary
    run's REVCON): the single point of the 90 CO2 it holds must equal the energy the unary run
    stored in its REVIVE for the same state, up to REVCON's 10 significant digits."""
    c = oracle_mod.Chain(decks["binary_preloaded"], seed=(12, 34, 56, 78))
    ref = expected()["revive_energy_kcal"]
    assert c.ints()["ntpguest"] == 2
    assert abs(c.scalars()["spenergy"] - ref) <= 1e-8 * abs(ref)


def test_single_point_deck_runs_no_moves(oracle_mod, tmp_path):
    """CONTROL without `steps` means a single point (readinputs.f: mcsteps 1, lspe): the
    reference computes the energy and stops before the move loop (gcmc.f:565-567); with `steps`
    the same deck runs until its cycles end."""
    import shutil

    calf = os.path.join(GOLDEN, "calf20")
    sp = tmp_path / "sp"
    shutil.copytree(calf, sp)
    ctl = [ln for ln in (sp / "CONTROL").read_text().split("\n") if not ln.startswith("steps")]
    (sp / "CONTROL").write_text("\n".join(ctl))
    a, b = oracle_mod.Chain(str(sp)), oracle_mod.Chain(calf)
    assert a.scalars()["spenergy"] == b.scalars()["spenergy"]
    assert a.run_to_completion(500) == 0
    assert b.run_to_completion(500) == 500


def test_tables_against_their_closed_forms(oracle_mod):
    """The two interpolation tables against the formulas they tabulate, on the CALF-20 deck
    (the product's tables equal the oracle's bit for bit, tests/test_host.py): erc(i) * r_i is
    A&S 7.1.26's erfc(alpha r_i) (erfcgen, ewald.f:1-30), within that approximation's published
    bound of 1.5e-7; every lj row of vvv is 4 eps [(sigma/r)^12 - (sigma/r)^6] in internal units
    (forgen, vdw_terms.f:238-250) at r_i = i * dlrpot."""
    import math

    c = oracle_mod.Chain(CALF)
    s = c.scalars()
    erc, a, dr = c.erc(), s["alpha"], s["drewd"]
    err = max(abs(erc[i] * i * dr - math.erfc(a * i * dr)) for i in range(1, len(erc)))
    assert 1e-9 < err <= 1.5e-7
    lines = open(os.path.join(CALF, "FIELD")).read().splitlines()
    i0 = next(i for i, ln in enumerate(lines) if ln.lower().startswith("vdw"))
    npair = int(lines[i0].split()[1])
    assert npair == 28
    for k in range(1, npair + 1):
        f = lines[i0 + k].split()
        assert f[2] == "lj"
        eps, sig = float(f[3]), float(f[4])
        v = c.vvv(k)
        r = np.arange(1, len(v)) * s["dlrpot"]
        ref = 4.0 * eps * ((sig / r) ** 12 - (sig / r) ** 6) * s["engunit"]
        assert np.all(np.abs(v[1:] - ref) <= 1e-11 * np.abs(ref)), k
