"""Probability plots on the GPU paths against the oracle's storeprob, on the reference's
probability-plot example (CO2 in CALF-20; plots of site 1 and of sites 2+3) with production
from the first move.  The plain path sums the weights in FP64 in the reference's order; the
batched path sums them in fixed point (2^-32) with integer atomics, so its grids match to
~1e-7 absolute whatever the order of the adds."""
import os
import shutil

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
PP = os.path.join(HERE, "golden", "probplot")


@pytest.fixture(scope="module")
def deck(tmp_path_factory):
    d = tmp_path_factory.mktemp("probplot")
    for f in ("FIELD", "CONFIG", "CONTROL"):
        shutil.copy(os.path.join(PP, f), d / f)
    ctl = (d / "CONTROL").read_text().replace("equilibration    100000", "equilibration    0")
    (d / "CONTROL").write_text(ctl)
    return str(d)


def test_plain_prob_grids_match_oracle(fmc, oracle_mod, deck, tmp_path):
    seed = (12, 34, 56, 78)
    c = fmc.Chain(deck, seed=seed)
    orc = oracle_mod.Chain(deck, seed=seed)
    c.run(700)
    orc.run(700)
    gd, go = c.prob(), orc.prob()
    assert gd.shape == go.shape and go.sum() > 0
    assert np.max(np.abs(gd - go)) <= 1e-9 * go.max()
    # each production move bins every molecule once per plot site
    c.write_prob(str(tmp_path))
    assert sorted(os.listdir(tmp_path)) == ["prob_guest01_prob_01.cube", "prob_guest01_prob_02.cube"]


def test_batch_prob_grids_match_oracle(fmc, oracle_mod, deck, tmp_path):
    seeds = [(12, 34, 56, 78), (1, 2, 3, 4)]
    b = fmc.Batch([deck, deck], seeds)
    b.run(400)
    b.run(300)
    for i, s in enumerate(seeds):
        orc = oracle_mod.Chain(deck, seed=s)
        orc.run(700)
        go, gb = orc.prob(), b.prob(i)
        assert go.sum() > 0
        assert np.max(np.abs(gb - go)) < 1e-6, i
    b.write_prob(0, str(tmp_path))
    assert len(os.listdir(tmp_path)) == 2
