"""The reference's other shipped examples replayed on the GPU paths against the oracle:
examples/advance/2 (CO2 + N2 in CALF-20 with probability plots and grid factors 2 2 2),
examples/advance/3 (guest-specific move probabilities and acceptance ratios inside the &guest
blocks, 4 A cutoff on the 44-atom cell) and examples/restart/2 (a binary CO2 + TIP4P-Ew run
started from the unary run's REVCON with 90 CO2 preloaded)."""
import numpy as np
import pytest

from test_gpu_plain import _compare_traces

pytestmark = pytest.mark.gpu

EXAMPLES = [("calf20_co2_n2", 1500), ("guest_moves", 2000), ("binary_preloaded", 800)]


@pytest.mark.parametrize("name,n", EXAMPLES)
def test_example_plain_replays_oracle(fmc, oracle_mod, decks, name, n):
    seed = (103, 112, 53, 153)
    c = fmc.Chain(decks[name], seed=seed)
    o = oracle_mod.Chain(decks[name], seed=seed)
    sp_o = o.scalars()["spenergy"]
    assert abs(c.info()["spenergy"] - sp_o) <= 1e-9 * max(1.0, abs(sp_o))
    _compare_traces(c.run(n), o.run(n))
    for g in range(c.info()["nspecies"]):
        gd, go = c.guest_coords(g), o.guest_coords(g)
        assert gd.shape == go.shape
        if gd.size:
            assert np.max(np.abs(gd - go)) < 1e-9


@pytest.mark.parametrize("name,n", EXAMPLES)
def test_example_batch_replays_oracle(fmc, oracle_mod, decks, name, n):
    seeds = [(103, 112, 53, 153), (12, 34, 56, 78)]
    b = fmc.Batch([decks[name]] * 2, seeds)
    tr, _ = b.run(n, trace=True)
    for i, s in enumerate(seeds):
        _compare_traces(tr[i], oracle_mod.Chain(decks[name], seed=s).run(n))
