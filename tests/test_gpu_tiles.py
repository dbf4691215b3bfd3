"""Tile shapes of the batched kernel (threads per chain, k-vectors per thread per trip of the
reciprocal loop ewald.f:145-331, neighbour candidates per trip of the real-space loop
ewald.f:656-690 / vdw_terms.f:455-495) and their autotuner.

Every tile must replay the oracle move for move (per-move dE within the energy-scale bar, the
same accept sequence), and the tiles of one thread count must agree bit for bit: they only
change how many terms a thread has in flight, not the order in which it adds them."""
import numpy as np
import pytest

from test_gpu_plain import _compare_traces

pytestmark = pytest.mark.gpu

NAMES = ["small", "ortho0", "mixture", "calf20", "imcon5"]
SEEDS = [(12, 34, 56, 78), (1, 2, 3, 4), (9, 10, 11, 12), (5, 6, 7, 8), (17, 19, 23, 29)]


def _tile_index(fmc, shape):
    return fmc.batch_tiles().index(shape)


@pytest.mark.parametrize("shape", [(128, 1, 1), (384, 2, 2), (256, 2, 2), (128, 2, 2)])
def test_non_default_tile_replays_oracle(fmc, oracle_mod, decks, shape):
    dirs = [decks[n] for n in NAMES]
    b = fmc.Batch(dirs, SEEDS)
    b.tile = _tile_index(fmc, shape)
    assert b.tile == _tile_index(fmc, shape)
    n1, n2 = 900, 600
    tr1, _ = b.run(n1, trace=True)
    tr2, _ = b.run(n2, trace=True)
    for i, (d, s) in enumerate(zip(dirs, SEEDS)):
        ref = oracle_mod.Chain(d, seed=s).run(n1 + n2)
        _compare_traces(np.concatenate([tr1[i], tr2[i]]), ref)


@pytest.mark.parametrize("threads", [128, 256, 384])
def test_tiles_of_one_thread_count_agree_bitwise(fmc, decks, threads):
    dirs = [decks[n] for n in NAMES]
    states, traces = [], []
    for t, shape in enumerate(fmc.batch_tiles()):
        if shape[0] != threads:
            continue
        b = fmc.Batch(dirs, SEEDS)
        b.tile = t
        tr, _ = b.run(1200, trace=True)
        traces.append(tr)
        states.append([b.state(i) for i in range(len(dirs))])
    assert len(states) == 4
    for other_tr, other_st in zip(traces[1:], states[1:]):
        for i in range(len(dirs)):
            assert np.array_equal(traces[0][i]["estep"], other_tr[i]["estep"])
            assert np.array_equal(traces[0][i]["accepted"], other_tr[i]["accepted"])
            for k in ("energy0", "N", "E", "nmol0"):
                assert states[0][i][k] == other_st[i][k], k


def test_profiling_needs_the_default_tile(fmc, decks):
    b = fmc.Batch([decks["small"]], [(1, 2, 3, 4)])
    b.tile = 4
    with pytest.raises(fmc.FastMCError):
        b.profile(True)
    b.tile = 0
    b.profile(True)
    with pytest.raises(fmc.FastMCError):
        b.tile = 4


def test_autotune_tiles_returns_a_timed_tile(fmc, decks):
    dirs = [decks[n] for n in NAMES] * 4
    seeds = [(i + 1, 2, 3, 4) for i in range(len(dirs))]
    tiles = [0, 1, 4, 8]
    best, ms = fmc.autotune_tiles(dirs, seeds, voxel_edge=2.0, tiles=tiles, warm_moves=200, moves=200)
    assert best in tiles
    assert sorted(ms) == sorted(tiles)
    assert all(v > 0 for v in ms.values())
    assert ms[best] == min(ms.values())
