"""The configurations bench.py times, replayed against the oracle move for move.

* The plain FP64 drop-in workload: the 3392-atom cubic framework (a = 51.664 A), CO2 at 1 bar,
  kmax 12 (K = 4192), with the bench's seed; 20,000 moves on the plain path and on two chains of
  the batched kernel, each split across launches.
* The batched FP64 workload's own chains (16 frameworks x 16 pressures, the bench's seeds): the
  largest-K framework at the lowest and highest pressure, a replicated supercell, a replicated
  10-bar chain and a mid-size framework, 12,000 moves each in one batch over three launches (the
  bench's step is 2,000 moves).

Bars as in test_gpu_plain: identical move sequence, random numbers and accept/reject; per-move dE
within 1e-9 of the move's energy scale plus the FP64 floor of the reciprocal difference
(2 eps E_recip, recip_floor: at K = 4192 a rotation of dE ~ 1e-5 kcal/mol differs by 1e-12
kcal/mol between any two summation orders); final guest coordinates within 1e-9 A."""
import os

import numpy as np
import pytest

from test_gpu_plain import _compare_traces, recip_floor

pytestmark = pytest.mark.gpu

# bench.py's plain-workload seed
PLAIN_SEED = (12, 34, 56, 78)
# chain index = framework * 16 + pressure index: framework 1 (K = 952, the largest) at 0.01 and 10
# bar, framework 6 (replicated along c, K = 176) at 0.4 bar, framework 0 (replicated along b) at
# 10 bar, framework 12 (2091 atoms) at 2.5 bar
BATCHED_CHAINS = [16, 31, 104, 15, 204]


def _same_guests(a, b):
    assert a.shape == b.shape
    if a.size:
        assert np.max(np.abs(a - b)) < 1e-9


def test_plain_workload_20k_moves_match_oracle(fmc, oracle_mod, decks):
    d = decks["large"]
    assert fmc.deck_inspect(d)["K"] == 4192
    c = fmc.Chain(d, seed=PLAIN_SEED)
    got = np.concatenate([c.run(5000) for _ in range(4)])
    orc = oracle_mod.Chain(d, seed=PLAIN_SEED)
    floor = recip_floor(d, orc.sk())
    ref = orc.run(20000)
    _compare_traces(got, ref, floor)
    assert np.sum(ref["accepted"] == 1) > 100 and ref["nmols_after"][-1] > 0
    _same_guests(c.guest_coords(0), orc.guest_coords(0))
    c.close()


def test_plain_workload_batched_20k_moves_match_oracle(fmc, oracle_mod, decks):
    d = decks["large"]
    seeds = [PLAIN_SEED, (3, 14, 15, 92)]
    b = fmc.Batch([d, d], seeds)
    tr = np.concatenate([b.run(5000, trace=True)[0] for _ in range(4)], axis=1)
    for i, s in enumerate(seeds):
        orc = oracle_mod.Chain(d, seed=s)
        floor = recip_floor(d, orc.sk())
        _compare_traces(tr[i], orc.run(20000), floor)
        _same_guests(b.guest_coords(i, 0), orc.guest_coords(0))
    b.close()


def test_batched_workload_chains_match_oracle(fmc, oracle_mod, tmp_path):
    from fastmc_b200 import synth

    dirs = synth.write_batched(str(tmp_path / "batched"), select=BATCHED_CHAINS)
    seeds = [synth.batched_seed(i) for i in BATCHED_CHAINS]
    infos = [fmc.deck_inspect(d) for d in dirs]
    assert infos[0]["K"] == 952 and infos[2]["K"] == 176
    b = fmc.Batch(dirs, seeds, voxel_edge=1.0)  # the edge the bench's autotuner picks
    tr = np.concatenate([b.run(4000, trace=True)[0] for _ in range(3)], axis=1)
    loaded = 0
    for i, (d, s) in enumerate(zip(dirs, seeds)):
        orc = oracle_mod.Chain(d, seed=s)
        ref = orc.run(12000)
        _compare_traces(tr[i], ref)
        _same_guests(b.guest_coords(i, 0), orc.guest_coords(0))
        loaded = max(loaded, int(ref["nmols_after"][-1]))
    assert loaded >= 20  # the 10-bar chains carry guest-guest pairs
    b.close()
