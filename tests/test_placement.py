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


_LIVENESS_PROBE = """
import datetime, json, os, sys
sys.path.insert(0, {pkg!r})
import torch.distributed as dist
from fastmc_b200 import placement

rank, port, scenario, out = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3], sys.argv[4]
t = datetime.timedelta(seconds=30)
store = dist.TCPStore("127.0.0.1", port, 2, is_master=(rank == 0), timeout=t)
dist.init_process_group("gloo", store=store, rank=rank, world_size=2, timeout=t)
live = placement.Liveness(store, rank, 2, timeout_s=3.0)
res = {{"rank": rank, "steps": []}}
try:
    for step in range(3):
        if step == 1 and scenario == "crash" and rank == 1:
            os._exit(3)                      # dies between steps without a word
        if step == 1 and scenario == "crash_store" and rank == 0:
            os._exit(3)                      # the rank that hosts the store dies
        if step == 1 and scenario == "leave" and rank == 1:
            live.leave(0)                    # stops after step 0, on purpose
            json.dump(res, open(out, "w"))
            os._exit(0)
        live.check_in(step)
        live.wait_all(step)
        res["steps"].append(step)
    res["all"] = placement.gather([(rank, rank * 10)], liveness=live)
    dist.destroy_process_group()
except placement.RankLost as e:
    res.update(lost=e.rank, at=e.step, left=e.left, msg=str(e))
json.dump(res, open(out, "w"))
os._exit(0)
"""


def _free_port():
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("scenario", ["healthy", "crash", "leave", "crash_store"])
def test_lost_rank_is_found_between_steps(tmp_path, scenario):
    """Two gloo ranks on CPU check in after every step through the process group's store.  A
    rank that dies between steps (or the one hosting the store) is reported on the other rank as
    RankLost naming it, after the check-in timeout; one that leaves on purpose is reported at
    once; with both alive the steps and the gather complete."""
    import subprocess
    import sys
    import time

    probe = tmp_path / "probe.py"
    probe.write_text(_LIVENESS_PROBE.format(pkg=os.path.join(ROOT, "fastmc-1.4.0_b200")))
    port = _free_port()
    env = dict(os.environ, GLOO_SOCKET_IFNAME="lo")
    t0 = time.monotonic()
    procs = [subprocess.Popen([sys.executable, str(probe), str(r), str(port), scenario, str(tmp_path / f"r{r}.json")],
                              env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE) for r in range(2)]
    codes = [p.wait(timeout=120) for p in procs]
    elapsed = time.monotonic() - t0
    res = {r: json.load(open(tmp_path / f"r{r}.json")) for r in range(2) if (tmp_path / f"r{r}.json").exists()}
    if scenario == "healthy":
        assert codes == [0, 0]
        for r in range(2):
            assert res[r]["steps"] == [0, 1, 2] and res[r]["all"] == [[0, 0], [1, 10]]
    elif scenario == "crash":
        assert codes[1] == 3 and 1 not in res
        assert res[0]["lost"] == 1 and res[0]["at"] == 1 and res[0]["left"] is False
        assert res[0]["steps"] == [0] and "did not check in" in res[0]["msg"]
    elif scenario == "leave":
        assert res[0]["lost"] == 1 and res[0]["left"] is True and "after step 0" in res[0]["msg"]
        assert res[0]["steps"] == [0]
    else:
        # the store goes with its host: the other rank may still be confirming step 0 then
        assert codes[0] == 3 and 0 not in res
        assert res[1]["lost"] == 0 and res[1]["at"] in (0, 1) and res[1]["steps"] == list(range(res[1]["at"]))
    assert elapsed < 90
