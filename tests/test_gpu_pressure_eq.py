"""Pressure equilibration (gcmc.f:637-696, 1796-1808) on the plain and batched GPU paths against
the oracle: the move sequence through the adjustments, the forced settling, the restart of the
move count and the switch to production, and the partial pressures the acceptance uses."""
import numpy as np
import pytest

from test_gpu_plain import _compare_traces

pytestmark = pytest.mark.gpu

N = 7200


def test_plain_pressure_equilibration_matches_oracle(fmc, oracle_mod, decks):
    seed = (12, 34, 56, 78)
    c = fmc.Chain(decks["pressure_eq"], seed=seed)
    o = oracle_mod.Chain(decks["pressure_eq"], seed=seed)
    for _ in range(N // 1200):
        _compare_traces(c.run(1200), o.run(1200))
        pc, tc = c.pressures()
        po, to = o.pressures()
        assert tc == to
        assert np.allclose(pc, po, rtol=1e-12, atol=0)
    assert to == 0.0  # settled within the run


def test_batch_pressure_equilibration_matches_oracle(fmc, oracle_mod, decks):
    seeds = [(12, 34, 56, 78), (5, 6, 7, 8)]
    b = fmc.Batch([decks["pressure_eq"]] * 2, seeds)
    tr1, _ = b.run(N // 2, trace=True)
    tr2, _ = b.run(N - N // 2, trace=True)
    tr = np.concatenate([tr1, tr2], axis=1)
    for i, s in enumerate(seeds):
        o = oracle_mod.Chain(decks["pressure_eq"], seed=s)
        _compare_traces(tr[i], o.run(N))
        pb, tb = b.pressures(i)
        po, to = o.pressures()
        assert tb == to == 0.0
        assert np.allclose(pb, po, rtol=1e-12, atol=0)
