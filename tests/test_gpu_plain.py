"""Plain FP64 GPU path against the oracle and the reference's known answers.

Tolerance (FP64 path): 1e-9 relative, the bar stated for total energy and per-move dE; the
move sequence (move type, molecule choice, accept/reject) must be identical."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
CALF = os.path.join(GOLDEN, "calf20")
REL = 1e-9


def expected():
    with open(os.path.join(CALF, "expected.json")) as f:
        return json.load(f)


def relerr(a, b, floor=1e-300):
    return abs(a - b) / max(abs(b), floor)


def test_calf20_empty_framework_energy_on_device(fmc, oracle_mod):
    c = fmc.Chain(CALF, seed=expected()["seed"])
    info = c.info()
    assert info["K"] == 870 and info["imcon"] == 3
    assert abs(info["dlpeng"] - expected()["dlpeng_empty_kcal"]) <= 5e-7
    orc = oracle_mod.Chain(CALF, seed=expected()["seed"])
    assert relerr(info["dlpeng"], orc.scalars()["dlpeng"]) < REL
    sk_d, sk_o = c.sk(), orc.sk()
    assert np.max(np.abs(sk_d - sk_o)) <= 1e-10 * np.max(np.abs(sk_o))


def test_revive_state_single_point_on_device(fmc, oracle_mod):
    c = fmc.Chain(CALF, seed=expected()["seed"])
    guests = np.load(os.path.join(CALF, "revive_guests.npy"))
    c.set_guests(0, guests)
    sp, dlp = c.single_point()
    ref = expected()["revive_energy_kcal"]
    assert relerr(sp, ref) < REL
    orc = oracle_mod.Chain(CALF, seed=expected()["seed"])
    orc.load_guests(0, guests.reshape(-1, 3))
    assert relerr(sp, orc.scalars()["spenergy"]) < REL
    assert relerr(dlp, orc.scalars()["dlpeng"]) < REL
    sk_d, sk_o = c.sk(), orc.sk()
    assert np.max(np.abs(sk_d - sk_o)) <= 1e-10 * np.max(np.abs(sk_o))


def _random_guest(rng, tmpl_xyz, cell):
    f = rng.uniform(0, 1, 3)
    com = f @ cell
    th = rng.uniform(0, 2 * np.pi)
    ax = rng.normal(size=3)
    ax /= np.linalg.norm(ax)
    K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    R = np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * K @ K
    return tmpl_xyz @ R.T + com


@pytest.mark.parametrize("deck", ["calf20", "small", "ortho0", "mixture"])
def test_trial_pass_energies_match_oracle(fmc, oracle_mod, decks, deck):
    d = decks[deck]
    c = fmc.Chain(d)
    orc = oracle_mod.Chain(d)
    if deck == "calf20":
        guests = np.load(os.path.join(CALF, "revive_guests.npy"))
        c.set_guests(0, guests)
        orc.load_guests(0, guests.reshape(-1, 3))
    rng = np.random.default_rng(5)
    cell = np.array([[orc.scalars()["volm"] ** (1 / 3), 0, 0]])  # unused placeholder
    from fastmc_b200 import _lib  # noqa: F401
    info = c.info()
    ng = info["nspecies"]
    # cell rows from the CONFIG header of the deck
    lines = open(os.path.join(d, "CONFIG")).read().split("\n")
    cell = np.array([[float(v) for v in lines[k].split()] for k in (2, 3, 4)])
    for g in range(ng):
        tmpl, q, typ, mass = orc.guest_template(g)
        for trial in range(6):
            xyz = _random_guest(rng, tmpl, cell)
            e_d = c.ewald1_guest(g, xyz, fmc.INSERT)
            e_o = orc.ewald1_guest(g, xyz, oracle_mod.MV_INSERT)
            assert relerr(e_d, e_o) < REL, (g, trial, e_d, e_o)
            snew_d, snew_o = c.sk(pending=True), orc.sk(new=True)
            assert np.max(np.abs(snew_d - snew_o)) <= 1e-10 * np.max(np.abs(snew_o))
            r2_d, rv_d = c.guest_realspace(g, xyz, -1)
            r2_o, rv_o = orc.realspace(g, xyz)
            scale = max(abs(r2_o), abs(rv_o), 1.0)
            assert abs(r2_d - r2_o) <= REL * max(abs(r2_o), 1e-6 * scale), (r2_d, r2_o)
            assert abs(rv_d - rv_o) <= REL * max(abs(rv_o), 1e-6 * scale), (rv_d, rv_o)


def recip_floor(deck, sk):
    """kcal/mol below which two FP64 evaluations of one move's dE cannot agree: the reference's
    reciprocal change is pref*sum_k akk|S_new|^2 - pref*sum_k akk|S_old|^2 (ewald.f:311-319), a
    difference of two sums each of the chain's reciprocal energy E_recip, so its last bits are
    2 * eps * E_recip whatever the order of the additions (1e-12 kcal/mol on the 3392-atom deck,
    E_recip = 17,171 kcal/mol; 1e-14 on CALF-20)."""
    import fastmc_b200 as fm

    info = fm.deck_inspect(deck)
    pref = 2.0 * (2.0 * np.pi / info["volm"]) * 138935.4835
    e_recip = pref * float(np.sum(info["akk"] * np.abs(sk) ** 2)) / 418.4
    return 2.0 * np.finfo(np.float64).eps * e_recip


def _compare_traces(tr_d, tr_o, floor=0.0):
    for key in ("mtype", "iguest", "randchoice", "accepted", "nmols_after"):
        bad = np.nonzero(tr_d[key] != tr_o[key])[0]
        assert bad.size == 0, f"{key} differs first at move {bad[:1]}"
    assert np.array_equal(tr_d["rande"], tr_o["rande"])
    # dE relative to the move's energy scale: a dE that nearly cancels its components carries
    # their rounding, so the scale is the larger of |dE|, the summed |components| (internal
    # units of 10 J/mol, 418.4 to a kcal/mol) and 1e-3 kcal/mol
    comp = (np.abs(tr_o["ewld1"]) + np.abs(tr_o["ewld2"]) + np.abs(tr_o["ewld3"]) + np.abs(tr_o["vdw"])) / 418.4
    scale = np.maximum(np.maximum(np.abs(tr_o["estep"]), comp), 1e-3)
    err = np.maximum(np.abs(tr_d["estep"] - tr_o["estep"]) - floor, 0.0) / scale
    assert err.max() < REL, f"max rel dE error {err.max():.3e} at move {int(err.argmax())}"
    # components are in internal units (10 J/mol); the floor is the same 1e-3 kcal/mol as dE's
    for key in ("ewld1", "ewld2", "vdw", "delrc"):
        s = np.maximum(np.abs(tr_o[key]), 1e-3 * 418.4)
        e = np.abs(tr_d[key] - tr_o[key]) / s
        assert e.max() < 1e-8, (key, e.max())
    assert np.allclose(tr_d["energy_after"], tr_o["energy_after"], rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("deck,n", [("small", 4000), ("mixture", 3000), ("ortho1", 2000), ("forms", 2000),
                                    ("jumps", 2500), ("multijump", 2500), ("imcon4", 2000), ("imcon5", 2000),
                                    ("imcon6", 2000), ("imcon7", 2000)])
def test_move_loop_matches_oracle_sequence(fmc, oracle_mod, decks, deck, n):
    seed = (31, 41, 59, 26)
    c = fmc.Chain(decks[deck], seed=seed)
    orc = oracle_mod.Chain(decks[deck], seed=seed)
    tr_d = c.run(n)
    tr_o = orc.run(n)
    _compare_traces(tr_d, tr_o)
    for g in range(c.info()["nspecies"]):
        gd, go = c.guest_coords(g), orc.guest_coords(g)
        assert gd.shape == go.shape
        if gd.size:
            assert np.max(np.abs(gd - go)) < 1e-9


def test_dropin_reject_keeps_and_commit_takes_s_new(fmc, oracle_mod, decks):
    """The call surface a Fortran move loop uses: ewald1_guest + guest_realspace for a trial,
    then reject (S(k) and the sites untouched) or commit (S(k) <- S_new, the molecule added)."""
    d = decks["small"]
    c = fmc.Chain(d)
    tmpl, _, _, _ = oracle_mod.Chain(d).guest_template(0)
    lines = open(os.path.join(d, "CONFIG")).read().split("\n")
    cell = np.array([[float(v) for v in lines[k].split()] for k in (2, 3, 4)])
    xyz = _random_guest(np.random.default_rng(11), tmpl, cell)
    s0 = c.sk()
    c.ewald1_guest(0, xyz, fmc.INSERT)
    c.guest_realspace(0, xyz, -1)
    pending = c.sk(pending=True)
    assert not np.array_equal(pending, s0)
    c.reject()
    assert np.array_equal(c.sk(), s0) and c.guest_coords(0).shape[0] == 0
    c.ewald1_guest(0, xyz, fmc.INSERT)
    c.commit(fmc.INSERT, 0, -1, xyz)
    assert np.array_equal(c.sk(), pending)
    g = c.guest_coords(0)
    assert g.shape[0] == 1 and np.allclose(g[0], xyz)
