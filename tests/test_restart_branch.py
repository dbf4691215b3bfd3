"""CONTROL `restart` (readinputs.f:604-608): the deck readers accept the directive, and the
branch a node continues from follows gcmc.f:353-394 with revscan (utility_pack.f:1819-1839,
`ls | grep -c branch` in the working directory) and revread's missing-file rule
(utility_pack.f:1855-1860).  Host only: no GPU."""
import os
import shutil

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CALF = os.path.join(HERE, "golden", "calf20")


def restart_deck(dst):
    """The CALF-20 deck with `restart` as CONTROL's first directive."""
    os.makedirs(dst, exist_ok=True)
    for f in ("FIELD", "CONFIG"):
        shutil.copy(os.path.join(CALF, f), os.path.join(dst, f))
    lines = open(os.path.join(CALF, "CONTROL")).read().splitlines(True)
    with open(os.path.join(dst, "CONTROL"), "w") as f:
        f.write(lines[0] + "restart\n" + "".join(lines[1:]))
    return str(dst)


def _branch(work, n, revive=True):
    d = os.path.join(work, "branch%02d" % n)
    os.makedirs(d, exist_ok=True)
    if revive:
        open(os.path.join(d, "REVIVE"), "wb").close()
    return d


def test_no_branches_start_from_config(fmc, tmp_path):
    work = restart_deck(tmp_path / "job")
    for node in (0, 3):
        b = fmc.restart_branch(work, node)
        assert b == {"revive": None, "outdir": os.path.join(work, "branch%02d" % (node + 1)), "prevnodes": 0}


def test_nodes_map_onto_previous_branches(fmc, tmp_path):
    work = restart_deck(tmp_path / "job")
    _branch(work, 1)
    _branch(work, 2)
    # nodes within the previous run read their own branch, later ones wrap: mod(idnode+1, prev)+1
    want = {0: 1, 1: 2, 2: 2, 3: 1, 4: 2}
    for node, src in want.items():
        b = fmc.restart_branch(work, node)
        assert b["prevnodes"] == 2
        assert b["revive"] == os.path.join(work, "branch%02d" % src, "REVIVE")
        assert b["outdir"] == os.path.join(work, "branch%02d" % (node + 1))


def test_fewer_nodes_than_branches_ignore_the_rest(fmc, tmp_path):
    work = restart_deck(tmp_path / "job")
    for n in (1, 2, 3):
        _branch(work, n)
    assert fmc.restart_branch(work, 0)["revive"] == os.path.join(work, "branch01", "REVIVE")
    assert fmc.restart_branch(work, 0)["prevnodes"] == 3


def test_missing_revive_means_config(fmc, tmp_path):
    work = restart_deck(tmp_path / "job")
    _branch(work, 1, revive=False)
    b = fmc.restart_branch(work, 0)
    assert b["revive"] is None and b["prevnodes"] == 1
    # node 1 of one previous branch wraps onto branch01, which has no REVIVE either
    assert fmc.restart_branch(work, 1)["revive"] is None


def test_branch_count_is_the_listing_count(fmc, tmp_path):
    """revscan counts every listed name containing "branch", files included (the reference's own
    comment warns of it); hidden names are not listed."""
    work = restart_deck(tmp_path / "job")
    _branch(work, 1)
    open(os.path.join(work, "branch_notes.txt"), "w").close()
    open(os.path.join(work, ".branchrc"), "w").close()
    b = fmc.restart_branch(work, 2)
    assert b["prevnodes"] == 2
    # mod(3, 2) + 1 = 2: branch02 does not exist, so node 2 starts from the CONFIG
    assert b["revive"] is None


def test_node_index_and_buffers_are_checked(fmc, tmp_path):
    import ctypes

    from fastmc_b200 import FastMCError, lib

    work = restart_deck(tmp_path / "job")
    with pytest.raises(FastMCError):
        fmc.restart_branch(work, 99)
    with pytest.raises(FastMCError):
        fmc.restart_branch(work, -1)
    small = ctypes.create_string_buffer(8)
    assert lib().fmc_restart_branch(work.encode(), 0, None, 0, small, 8, None) < 0
    assert lib().fmc_restart_branch(work.encode(), 0, None, 0, None, 0, None) == 0


def test_readers_accept_the_directive(fmc, oracle_mod, tmp_path):
    """The directive changes no table: the product's host tables and the oracle's single point of
    the deck are those of the deck without it."""
    work = restart_deck(tmp_path / "job")
    a, b = fmc.deck_inspect(work), fmc.deck_inspect(CALF)
    for k in ("lmn", "akk", "erc", "charges"):
        assert np.array_equal(a[k], b[k])
    sa = oracle_mod.Chain(work, seed=(1, 2, 3, 4)).scalars()
    sb = oracle_mod.Chain(CALF, seed=(1, 2, 3, 4)).scalars()
    assert sa["spenergy"] == sb["spenergy"]
