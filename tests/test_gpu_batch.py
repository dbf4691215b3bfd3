"""Batched persistent kernel (FP64) against the oracle, chain by chain.

Each chain of a batch must reproduce the oracle's move sequence exactly (move type, species,
molecule choice, random numbers, accept/reject) with per-move dE within 1e-9 relative, whatever
else shares the launch."""
import numpy as np
import pytest

from test_gpu_plain import _compare_traces

pytestmark = pytest.mark.gpu


def test_batch_chains_replay_oracle(fmc, oracle_mod, decks):
    names = ["small", "ortho0", "ortho1", "mixture", "small", "ortho2"]
    seeds = [(12, 34, 56, 78), (1, 2, 3, 4), (5, 6, 7, 8), (9, 10, 11, 12), (31, 41, 59, 26), (17, 19, 23, 29)]
    dirs = [decks[n] for n in names]
    b = fmc.Batch(dirs, seeds)
    n1, n2 = 1200, 800
    tr1, _ = b.run(n1, trace=True)
    tr2, _ = b.run(n2, trace=True)  # state carries over between launches
    for i, (d, s) in enumerate(zip(dirs, seeds)):
        orc = oracle_mod.Chain(d, seed=s)
        ref = orc.run(n1 + n2)
        got = np.concatenate([tr1[i], tr2[i]])
        _compare_traces(got, ref)
        st = b.state(i)
        assert st["status"] == 0
        assert st["moves"] == n1 + n2
        go = orc.guest_coords(0)
        gb = b.guest_coords(i, 0)
        assert gb.shape == go.shape
        if gb.size:
            assert np.max(np.abs(gb - go)) < 1e-9


def test_batch_isolation_alone_vs_mixed(fmc, decks):
    """A chain gives the same trajectory alone and inside a mixed batch."""
    seed = (3, 1, 4, 1)
    alone = fmc.Batch([decks["ortho1"]], [seed])
    ta, _ = alone.run(1000, trace=True)
    mixed = fmc.Batch([decks["small"], decks["ortho1"], decks["mixture"]], [(7, 7, 7, 7), seed, (8, 8, 8, 8)])
    tm, _ = mixed.run(1000, trace=True)
    for key in ("mtype", "randchoice", "accepted", "nmols_after"):
        assert np.array_equal(ta[0][key], tm[1][key])
    assert np.array_equal(ta[0]["estep"], tm[1]["estep"])


def test_batch_every_vdw_form_replays_oracle(fmc, oracle_mod, decks):
    """All nine pair forms of forgen in one deck (each pair of types uses one of them)."""
    seeds = [(2, 4, 6, 8), (3, 5, 7, 9)]
    b = fmc.Batch([decks["forms"]] * 2, seeds)
    tr, _ = b.run(1500, trace=True)
    for i, s in enumerate(seeds):
        _compare_traces(tr[i], oracle_mod.Chain(decks["forms"], seed=s).run(1500))


def test_batch_jump_flex_swap_replay_oracle(fmc, oracle_mod, decks):
    """Long jumps (gcmc.f:1389-1547) and the flex / swap moves the reference selects but does not
    implement, mixed with insertions, deletions, displacements and rotations."""
    seeds = [(4, 8, 15, 16), (23, 42, 4, 8)]
    b = fmc.Batch([decks["jumps"]] * 2, seeds)
    tr, _ = b.run(2500, trace=True)
    accepted_jumps = 0
    for i, s in enumerate(seeds):
        ref = oracle_mod.Chain(decks["jumps"], seed=s).run(2500)
        _compare_traces(tr[i], ref)
        assert np.any(ref["mtype"] == fmc.JUMP) and np.any(ref["mtype"] == fmc.NOOP)
        accepted_jumps += int(np.sum((ref["mtype"] == fmc.JUMP) & (ref["accepted"] == 1)))
    assert accepted_jumps > 0


def test_batch_multi_jump_replays_oracle(fmc, oracle_mod, decks):
    """Multiple long jumps (gcmc.f:1557-1785): the first jump is committed inside the launch while
    the second is evaluated, and a rejection restores S(k) and the first molecule; the trace,
    energies and final coordinates follow the oracle over launches that end mid-run."""
    seeds = [(4, 8, 15, 16), (23, 42, 4, 8), (1, 2, 3, 4)]
    b = fmc.Batch([decks["multijump"]] * 3, seeds)
    tr1, _ = b.run(1300, trace=True)
    tr2, _ = b.run(1200, trace=True)
    tr = np.concatenate([tr1, tr2], axis=1)
    acc_mj = rej_mj = 0
    for i, s in enumerate(seeds):
        orc = oracle_mod.Chain(decks["multijump"], seed=s)
        ref = orc.run(2500)
        _compare_traces(tr[i], ref)
        mj = ref["mtype"] == fmc.MULTIJUMP
        acc_mj += int(np.sum(mj & (ref["accepted"] == 1)))
        rej_mj += int(np.sum(mj & (ref["accepted"] == 0)))
        st = b.state(i)
        assert st["nmol0"] == ref["nmols_after"][-1]
        assert abs(st["energy0"] - ref["energy_after"][-1]) <= 1e-9 * max(1.0, abs(ref["energy_after"][-1]))
    assert acc_mj > 0 and rej_mj > 0


@pytest.mark.parametrize("name", ["imcon4", "imcon5", "imcon6", "imcon7"])
def test_batch_half_shift_cells_replay_oracle(fmc, oracle_mod, decks, name):
    """Truncated octahedron, rhombic dodecahedron and hexagonal prism cells: the images of
    utility_pack.f:1203-1346 in the real-space loop, voxel lists built over the box with the
    half-shift lattice's nearest images."""
    seeds = [(31, 41, 59, 26), (2, 7, 1, 8)]
    b = fmc.Batch([decks[name]] * 2, seeds)
    tr, _ = b.run(2000, trace=True)
    for i, s in enumerate(seeds):
        _compare_traces(tr[i], oracle_mod.Chain(decks[name], seed=s).run(2000))


def test_batch_finer_voxels_replay_oracle(fmc, oracle_mod, decks):
    """Neighbour lists over 1 A voxels (the autotuner's finest candidate) give the same moves."""
    seeds = [(9, 9, 9, 9), (10, 20, 30, 40)]
    names = ["ortho0", "mixture"]
    b = fmc.Batch([decks[n] for n in names], seeds, voxel_edge=1.0)
    tr, _ = b.run(1500, trace=True)
    for i, (n, s) in enumerate(zip(names, seeds)):
        _compare_traces(tr[i], oracle_mod.Chain(decks[n], seed=s).run(1500))


def test_voxel_autotune_returns_a_candidate(fmc, decks):
    dirs = [decks["ortho0"], decks["ortho1"]]
    edge, ms = fmc.autotune_voxel_edge(dirs, edges=(2.0, 1.25), moves=200)
    assert edge in (2.0, 1.25) and set(ms) == {2.0, 1.25} and all(v > 0 for v in ms.values())
    assert ms[edge] == min(ms.values())
