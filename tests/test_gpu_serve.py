"""Serving with continuous batching: requests admitted into free slots as others retire.

A served request must end in exactly the state the same deck and seed reach in a batch of
their own (FP64: nmol, energies and production statistics bitwise), whatever the other
requests in the launches were and however the move budget was cut into steps.  Steps are
pipelined: a step queues the next launch and then completes the previous one, so results, polls
and cancellations refer to the last completed launch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REQS = [("small", (12, 34, 56, 78), 1700), ("ortho0", (1, 2, 3, 4), 900), ("mixture", (9, 10, 11, 12), 2300),
        ("ortho1", (5, 6, 7, 8), 600), ("small", (31, 41, 59, 26), 1250), ("ortho2", (17, 19, 23, 29), 1000),
        ("ortho0", (2, 7, 1, 8), 400)]


def _alone(fmc, d, seed, moves):
    b = fmc.Batch([d], [seed])
    b.run(moves)
    return b.state(0)


def _same(res, st):
    assert res["moves"] == st["moves"]
    for g in range(4):
        assert res[f"nmol{g}"] == st[f"nmol{g}"]
        assert res[f"energy{g}"] == st[f"energy{g}"]
    for k in ("prodcount", "N", "E", "EN", "N2", "E2", "accept_ins", "accept_del"):
        assert res[k] == st[k], k


def test_continuous_batching_matches_isolated_runs(fmc, decks):
    srv = fmc.Server(slots=3, k_capacity=2400)
    ids = [srv.submit(decks[n], s, m) for n, s, m in REQS]
    seen_active, steps, finished = [], 0, []
    while srv.busy():
        active, queued, ms = srv.step(250)
        finished += srv.poll_done()
        steps += 1
        seen_active.append(active)
        assert active <= 3
        assert steps < 100
    # more requests than slots: later requests waited for retirements
    assert max(seen_active) == 3
    assert sorted(f[0] for f in finished) == sorted(ids)
    assert all(f[1] == srv.DONE and f[2]["moves"] == REQS[ids.index(f[0])][2] for f in finished)
    for rid, (n, s, m) in zip(ids, REQS):
        res = srv.poll(rid)
        assert res["state"] == srv.DONE, res
        assert res["moves"] == m and res["budget"] == m
        _same(res, _alone(fmc, decks[n], s, m))
    used, budget = srv.memory()
    assert used == 0 and budget > 0


def test_serve_cancel_and_reject(fmc, decks, tmp_path):
    # k capacity below the small deck's K: that request is rejected at admission
    k_cap = fmc.deck_inspect(decks["ortho0"])["K"]
    assert fmc.deck_inspect(decks["small"])["K"] > k_cap
    srv = fmc.Server(slots=2, k_capacity=k_cap)
    big = srv.submit(decks["small"], (1, 2, 3, 4), 100)
    missing = srv.submit(str(tmp_path / "no_such_deck"), (1, 1, 1, 1), 100)
    a = srv.submit(decks["ortho0"], (12, 34, 56, 78), 800)
    b = srv.submit(decks["ortho0"], (31, 41, 59, 26), 5000)
    c = srv.submit(decks["ortho0"], (5, 5, 5, 5), 300)
    srv.cancel(c)  # cancelled while queued: never runs
    srv.step(200)  # admits a and b and queues their first launch
    assert srv.poll(missing)["state"] == srv.REJECTED
    r = srv.poll(big)
    assert r["state"] == srv.REJECTED and "k-vector" in r["error"]
    assert srv.poll(a)["state"] == srv.RUNNING and srv.poll(b)["state"] == srv.RUNNING
    srv.step(200)  # queues the second launch, completes the first
    srv.cancel(b)  # cancelled while its second launch runs: switched off, last completed state kept
    rb = srv.poll(b)
    assert rb["state"] == srv.CANCELLED and rb["moves"] == 200
    done = [f[0] for f in srv.poll_done()]
    assert set(done) == {c, big, missing, b}
    while srv.busy():
        srv.step(200)
    assert srv.poll(c)["state"] == srv.CANCELLED and srv.poll(c)["moves"] == 0
    ra = srv.poll(a)
    assert ra["state"] == srv.DONE
    _same(ra, _alone(fmc, decks["ortho0"], (12, 34, 56, 78), 800))


def test_serve_memory_budget_limits_admission(fmc, decks):
    """A budget that holds one slot admits one request at a time; a request larger than the
    whole budget is rejected."""
    probe = fmc.Server(slots=1)
    probe.submit(decks["small"], (1, 2, 3, 4), 10**6)
    probe.step(1)
    slot_bytes, _ = probe.memory()
    probe.close()
    assert slot_bytes > 0
    srv = fmc.Server(slots=4, mem_budget=int(1.5 * slot_bytes))
    ids = [srv.submit(decks["small"], (i + 1, 2, 3, 4), 300) for i in range(3)]
    active_seen = []
    for _ in range(40):
        if not srv.busy():
            break
        active, queued, _ = srv.step(300)
        active_seen.append(active)
        used, budget = srv.memory()
        assert used <= budget
    assert all(srv.poll(i)["state"] == srv.DONE for i in ids)
    assert max(active_seen) == 1
    tiny = fmc.Server(slots=2, mem_budget=1 << 20)
    rid = tiny.submit(decks["small"], (1, 2, 3, 4), 100)
    tiny.step(100)
    r = tiny.poll(rid)
    assert r["state"] == tiny.REJECTED and "memory budget" in r["error"]


def test_serve_deck_cycle_budget_matches_oracle(fmc, oracle_mod, tmp_path):
    """moves=0: a request runs until its deck's own equilibration + production cycles end, on
    the same move as the reference loop (gcmc.f:594-736), with the same statistics."""
    from fastmc_b200 import synth

    d = synth.write_plain_small(str(tmp_path / "short"), cycles=3)
    seed = (12, 34, 56, 78)
    orc = oracle_mod.Chain(d, seed=seed)
    n_ref = orc.run_to_completion(10**6)
    assert 2000 < n_ref < 10**6
    srv = fmc.Server(slots=2)
    rid = srv.submit(d, seed)
    other = srv.submit(d, (1, 2, 3, 4), 700)
    for _ in range(200):
        if not srv.busy():
            break
        srv.step(900)
    res = srv.poll(rid)
    assert res["state"] == srv.DONE and res["finished"] == 1.0
    assert res["moves"] == n_ref
    ref = orc.stats(0)
    assert res["prodcount"] == ref["prodcount"]
    for k in ("N", "E", "EN", "N2", "E2"):
        assert abs(res[k] - ref[k]) <= 1e-8 * max(abs(ref[k]), 1.0), k
    assert srv.poll(other)["moves"] == 700 and srv.poll(other)["finished"] == 0.0


def test_serve_starts_from_preloaded_guests_and_a_revive(fmc, decks, tmp_path):
    """Requests that start with guests -- the deck's own (FIELD NUMMOLS > 0: the reference's
    binary CO2 + TIP4P-Ew deck on 90 CO2) or a REVIVE's (CONTROL `restart` with branch01/REVIVE
    beside the CALF-20 deck, gcmc.f:353-418) -- end in the state the same deck and seed reach in
    a batch of their own, beside a request from the empty framework and across steps."""
    import json
    import os

    from test_restart_branch import CALF, restart_deck

    exp = json.load(open(os.path.join(CALF, "expected.json")))
    guests = np.load(os.path.join(CALF, "revive_guests.npy"))
    work = restart_deck(tmp_path / "job")
    os.makedirs(os.path.join(work, "branch01"))
    fmc.write_revive_state(CALF, os.path.join(work, "branch01"), [guests], production=True,
                           chainstats=exp["revive_chainstats"], energy=[exp["revive_energy_kcal"]])
    reqs = [(work, (103, 112, 53, 153), 900), (decks["binary_preloaded"], (1, 2, 3, 4), 700),
            (decks["ortho0"], (5, 6, 7, 8), 500)]
    srv = fmc.Server(slots=2, k_capacity=2400)
    ids = [srv.submit(d, s, m) for d, s, m in reqs]
    for _ in range(100):
        if not srv.busy():
            break
        srv.step(300)
    for rid, (d, s, m) in zip(ids, reqs):
        res = srv.poll(rid)
        assert res["state"] == srv.DONE, res
        _same(res, _alone(fmc, d, s, m))
    assert srv.poll(ids[0])["nmol0"] > 0 and srv.poll(ids[1])["nmol0"] > 0


def test_serve_checkpoint_of_a_finished_request_resumes(fmc, decks, tmp_path):
    """A finished request's REVIVE / REVCON (final state kept at retirement) are byte for byte the
    files the same deck and seed write after the same moves in a batch of their own, and a
    request on the deck with CONTROL `restart` and that REVIVE resumes as the batch does."""
    import os
    import shutil

    d, seed, m = decks["ortho0"], (12, 34, 56, 78), 900
    srv = fmc.Server(slots=2)
    srv.keep_final_state(True)
    rid = srv.submit(d, seed, m)
    other = srv.submit(d, (1, 2, 3, 4), 1300)
    cancelled = srv.submit(d, (4, 3, 2, 1), 5000)
    srv.cancel(cancelled)
    for _ in range(100):
        if not srv.busy():
            break
        srv.step(400)
    got, ref = tmp_path / "served", tmp_path / "batch"
    os.makedirs(got)
    os.makedirs(ref)
    srv.write_revive(rid, got)
    b = fmc.Batch([d], [seed])
    b.run(m)
    b.write_revive(0, str(ref))
    for f in ("REVIVE", "REVCON"):
        assert (got / f).read_bytes() == (ref / f).read_bytes(), f
    with pytest.raises(fmc.FastMCError):
        srv.write_revive(cancelled, tmp_path)
    # resume: the deck with `restart` and the served REVIVE as branch01/REVIVE
    job = tmp_path / "resume"
    shutil.copytree(d, job)
    ctl = (job / "CONTROL").read_text().split("\n")
    (job / "CONTROL").write_text("\n".join([ctl[0], "restart"] + ctl[1:]))
    os.makedirs(job / "branch01")
    shutil.copy(got / "REVIVE", job / "branch01" / "REVIVE")
    again = srv.submit(str(job), (7, 7, 7, 7), 600)
    for _ in range(100):
        if not srv.busy():
            break
        srv.step(400)
    res = srv.poll(again)
    assert res["state"] == srv.DONE and res["nmol0"] > 0
    _same(res, _alone(fmc, str(job), (7, 7, 7, 7), 600))
    assert srv.poll(other)["state"] == srv.DONE
