"""numguests.out and his.xyz of the plain and batched GPU paths against the oracle's files on
the same deck and seed (CO2 + N2 mixture: one file per species).  The integer columns must be
equal; the printed energies agree to one unit of the last printed decimal."""
import os

import numpy as np
import pytest

from test_outputs import read_numguests, with_outputs

pytestmark = pytest.mark.gpu


def _same_numguests(a, b):
    ra, rb = read_numguests(a), read_numguests(b)
    assert len(ra) == len(rb) > 0
    for x, y in zip(ra, rb):
        assert x[0:2] == y[0:2] and x[4:] == y[4:], (x, y)
        assert abs(x[2] - y[2]) <= 1.5e-6 and abs(x[3] - y[3]) <= 1.5e-6, (x, y)


def _same_xyz(a, b):
    la, lb = open(a).read().split("\n"), open(b).read().split("\n")
    assert len(la) == len(lb) > 2
    for x, y in zip(la, lb):
        if x.startswith("  ") and len(x) > 3:
            assert x[:3] == y[:3]
            assert np.allclose([float(v) for v in x[3:].split()], [float(v) for v in y[3:].split()], atol=1.5e-6)
        else:
            assert x == y


def test_plain_chain_trajectory_files_match_oracle(fmc, oracle_mod, decks, tmp_path):
    deck = with_outputs(decks["mixture"], str(tmp_path / "deck"), 7, -50)
    seed = (12, 34, 56, 78)
    od, gd = tmp_path / "oracle", tmp_path / "gpu"
    od.mkdir()
    gd.mkdir()
    o = oracle_mod.Chain(deck, seed=seed)
    o.open_outputs(str(od))
    o.run(1500)
    o.open_outputs(None)
    c = fmc.Chain(deck, seed=seed)
    c.open_outputs(str(gd))
    c.run(1500)
    c.open_outputs(None)
    assert sorted(os.listdir(gd)) == sorted(os.listdir(od))
    for g in (1, 2):
        _same_numguests(gd / f"numguests0{g}.out", od / f"numguests0{g}.out")
        _same_xyz(gd / f"his0{g}.xyz", od / f"his0{g}.xyz")


def test_batch_numguests_from_trace_matches_oracle(fmc, oracle_mod, decks, tmp_path):
    deck = with_outputs(decks["mixture"], str(tmp_path / "deck"), 7, 0)
    seeds = [(12, 34, 56, 78), (9, 8, 7, 6)]
    b = fmc.Batch([deck, deck], seeds)
    gd = [tmp_path / "gpu0", tmp_path / "gpu1"]
    for d in gd:
        d.mkdir()
    for part, moves in enumerate((800, 700)):
        tr, _ = b.run(moves, trace=True)
        for i in range(2):
            b.write_numguests(i, tr, str(gd[i]), append=part > 0)
    for i, s in enumerate(seeds):
        od = tmp_path / f"oracle{i}"
        od.mkdir()
        o = oracle_mod.Chain(deck, seed=s)
        o.open_outputs(str(od))
        o.run(1500)
        o.open_outputs(None)
        for g in (1, 2):
            _same_numguests(gd[i] / f"numguests0{g}.out", od / f"numguests0{g}.out")
