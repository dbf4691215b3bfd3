"""The first 1e5 moves of a chain on the 424-atom cubic framework (CO2 at 0.15 bar), plain and
batched, against the oracle: the move types, molecule choices, random numbers and the FP64
accept/reject sequence identical move for move, dE within 1e-9 of each move's energy scale."""
import numpy as np
import pytest

from test_gpu_plain import _compare_traces

pytestmark = pytest.mark.gpu

N = 100_000


def test_plain_first_1e5_moves_match_oracle(fmc, oracle_mod, decks):
    seed = (12, 34, 56, 78)
    c = fmc.Chain(decks["small"], seed=seed)
    o = oracle_mod.Chain(decks["small"], seed=seed)
    for _ in range(4):
        _compare_traces(c.run(N // 4), o.run(N // 4))
    gd, go = c.guest_coords(0), o.guest_coords(0)
    assert gd.shape == go.shape and np.max(np.abs(gd - go)) < 1e-9


def test_batch_first_1e5_moves_match_oracle(fmc, oracle_mod, decks):
    seeds = [(12, 34, 56, 78), (103, 112, 53, 153)]
    b = fmc.Batch([decks["small"]] * 2, seeds)
    oracles = [oracle_mod.Chain(decks["small"], seed=s) for s in seeds]
    for _ in range(4):
        tr, _ = b.run(N // 4, trace=True)
        for i, o in enumerate(oracles):
            _compare_traces(tr[i], o.run(N // 4))
    for i, o in enumerate(oracles):
        assert b.state(i)["nmol0"] == o.guest_coords(0).shape[0]
