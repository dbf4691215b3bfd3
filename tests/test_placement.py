"""Placement of independent chains on GPUs by work and device memory (CPU only), and the
two-rank flow over gloo: every rank computes the same partition, runs its share and the results
are gathered once at the end."""
import json
import os
import textwrap

import pytest

from test_multiproc import ROOT, _torchrun


def test_assign_balances_work_and_respects_memory(fmc):
    from fastmc_b200 import placement

    work = [10, 9, 8, 7, 6, 5, 4, 3, 2, 1, 1, 1]
    p = placement.assign(work, 3)
    assert sorted(set(p)) == [0, 1, 2] and len(p) == len(work)
    load = [sum(w for w, g in zip(work, p) if g == k) for k in range(3)]
    assert max(load) - min(load) <= max(work)
    # memory: two large items cannot share a GPU of 10 units
    sizes = [6, 6, 1, 1]
    p = placement.assign([1, 1, 1, 1], 2, sizes=sizes, capacity=10)
    assert p[0] != p[1]
    for g in range(2):
        assert sum(s for s, q in zip(sizes, p) if q == g) <= 10
    with pytest.raises(ValueError):
        placement.assign([1], 2, sizes=[11], capacity=10)
    # deterministic: the same inputs give the same partition on every rank
    assert placement.assign(work, 3) == placement.assign(list(work), 3)


def test_footprint_grows_with_the_framework(fmc, decks):
    from fastmc_b200 import placement

    small_b, small_c = placement.footprint(decks["small"])
    large_b, large_c = placement.footprint(decks["large"])
    assert 0 < small_b < large_b
    assert 0 < small_c < large_c


def test_two_ranks_place_run_and_gather(tmp_path):
    probe = tmp_path / "probe.py"
    probe.write_text(textwrap.dedent(f"""
        import json, sys
        sys.path.insert(0, {ROOT!r})
        sys.path.insert(0, {os.path.join(ROOT, "fastmc-1.4.0_b200")!r})
        import bench
        from fastmc_b200 import placement
        d = bench.Dist(2)
        work = [5.0, 3.0, 8.0, 1.0, 2.0, 7.0, 4.0]
        p = placement.assign(work, d.world)
        mine = placement.share(work, p, d.rank)
        done = [(i, w * 10.0) for i, w in mine]   # stands in for running the chains
        allres = placement.gather(done)
        out = {{"rank": d.rank, "mine": [i for i, _ in mine], "all": allres}}
        with open({str(tmp_path)!r} + f"/rank{{d.rank}}.json", "w") as f:
            json.dump(out, f)
        d.close()
    """))
    r = _torchrun([str(probe)], timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    # one file per rank (the ranks' stdout lines may interleave)
    res = [json.load(open(tmp_path / f"rank{k}.json")) for k in range(2)]
    assert sorted(x["rank"] for x in res) == [0, 1]
    mine = sorted(i for x in res for i in x["mine"])
    assert mine == list(range(7))  # every item on exactly one rank
    for x in res:
        assert [i for i, _ in x["all"]] == list(range(7))
        assert [v for _, v in x["all"]] == [w * 10.0 for w in [5.0, 3.0, 8.0, 1.0, 2.0, 7.0, 4.0]]
