"""Mixed-precision batched path against the FP64 batched path (itself checked against the oracle).

Mixed precision evaluates phases and pair terms in FP32, keeps S(k), totals and the dE
assembly in FP64, and re-evaluates in FP64 any move whose acceptance margin lies inside the
FP32 error band.  Therefore the move sequence must be the FP64 sequence exactly (tested on
every move).  The dE error against FP64 on the same state (shadow run) is measured per
component; relative to max(|dE_fp64|, 1 kcal/mol) it reaches ~1.4e-4 with FP32 reciprocal
phases, ~2e-5 with FP32 Coulomb and ~1e-5 with FP32 vdW pair terms (the 1e-6 goal is not met
by FP32 terms; FP64 is the default).  The bars below sit above those measurements.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
DE_REL = {7: 5e-4, 4: 5e-5}  # all components FP32; vdW pair terms only


def _decks(decks):
    names = ["mixture", "ortho0", "ortho1", "small"]
    seeds = [(9, 10, 11, 12), (1, 2, 3, 4), (5, 6, 7, 8), (12, 34, 56, 78)]
    return [decks[n] for n in names], seeds


def test_mixed_follows_fp64_sequence(fmc, decks):
    dirs, seeds = _decks(decks)
    b64 = fmc.Batch(dirs, seeds)
    bmx = fmc.Batch(dirs, seeds)
    bmx.set_precision(7, recompute_every=1000)
    n = 3000
    t64, _ = b64.run(n, trace=True)
    tmx, _ = bmx.run(n, trace=True)
    for i in range(len(dirs)):
        for key in ("mtype", "iguest", "randchoice", "accepted", "nmols_after"):
            assert np.array_equal(t64[i][key], tmx[i][key]), (i, key)
        assert np.array_equal(t64[i]["rande"], tmx[i]["rande"])
        err = np.abs(tmx[i]["estep"] - t64[i]["estep"]) / np.maximum(np.abs(t64[i]["estep"]), 1.0)
        assert err.max() < DE_REL[7], (i, err.max())
        # running energy (the FP64 accumulator of accepted dE) stays within the same bar
        e64, emx = t64[i]["energy_after"][-1], tmx[i]["energy_after"][-1]
        assert abs(emx - e64) <= DE_REL[7] * max(abs(e64), 1.0) * 10
    st = bmx.state(0)
    assert st["recomputes"] >= 1


@pytest.mark.parametrize("mask", [7, 4])
def test_mixed_shadow_error_on_same_state(fmc, decks, mask):
    dirs, seeds = _decks(decks)
    bmx = fmc.Batch(dirs, seeds)
    bmx.run(1500)
    bmx.set_precision(mask, recompute_every=0)
    rec, sh, _ = bmx.run_shadow(1500)
    for i in range(len(dirs)):
        mixed = rec[i]["estep"]
        # moves decided after an FP64 re-evaluation report the FP64 value itself
        m = rec[i]["pad0"] == 0
        err = np.abs(mixed[m] - sh[i][m, 3]) / np.maximum(np.abs(sh[i][m, 3]), 1.0)
        assert err.max() < DE_REL[mask], (i, err.max())
        assert np.all(mixed[~m] == sh[i][~m, 3])
