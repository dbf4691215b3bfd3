"""Restart from a REVIVE (gcmc.f:353-418 with revread) on the plain and batched paths, and
checkpoints written by the batched path that restart elsewhere.

The REVIVE used here is the reference's CALF-20 90-CO2 state (written by the byte-exact writer
from the golden fixture).  After a restart the move sequence must be the oracle's after the same
restart (guests loaded, fresh single point, production flag and chain statistics restored)."""
import json
import os
import shutil

import numpy as np
import pytest

from test_gpu_plain import REL, _compare_traces

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CALF = os.path.join(HERE, "golden", "calf20")
SEED = (103, 112, 53, 153)


@pytest.fixture(scope="module")
def revive(fmc, tmp_path_factory):
    exp = json.load(open(os.path.join(CALF, "expected.json")))
    guests = np.load(os.path.join(CALF, "revive_guests.npy"))
    d = tmp_path_factory.mktemp("revive")
    fmc.write_revive_state(CALF, str(d), [guests], production=True, chainstats=exp["revive_chainstats"],
                           energy=[exp["revive_energy_kcal"]])
    return str(d / "REVIVE"), guests, exp


def _oracle_restart(oracle_mod, guests, exp, seed=SEED):
    orc = oracle_mod.Chain(CALF, seed=seed)
    orc.load_guests(0, guests.reshape(-1, 3))
    orc.restart_flags(True, np.asarray(exp["revive_chainstats"]))
    return orc


def test_plain_restart_follows_oracle(fmc, oracle_mod, revive):
    path, guests, exp = revive
    c = fmc.Chain(CALF, seed=SEED)
    c.restart(path)
    orc = _oracle_restart(oracle_mod, guests, exp)
    sp = c.info()["spenergy"]
    assert abs(sp - orc.scalars()["spenergy"]) <= REL * abs(sp)
    assert abs(sp - exp["revive_energy_kcal"]) <= 1e-9 * abs(sp)
    _compare_traces(c.run(600), orc.run(600))
    assert abs(c.stats(0)["N"] - orc.stats(0)["N"]) <= 1e-9 * orc.stats(0)["N"]


def test_batch_restart_follows_oracle(fmc, oracle_mod, revive):
    path, guests, exp = revive
    b = fmc.Batch([CALF, CALF], [SEED, (1, 2, 3, 4)])
    b.restart(0, path)
    st = b.state(0)
    assert st["nmol0"] == len(guests) and b.state(1)["nmol0"] == 0
    assert abs(st["energy0"] - exp["revive_energy_kcal"]) <= 1e-9 * abs(st["energy0"])
    orc = _oracle_restart(oracle_mod, guests, exp)
    tr, _ = b.run(800, trace=True)
    _compare_traces(tr[0], orc.run(800))


def test_batch_checkpoint_restarts_on_the_plain_path(fmc, oracle_mod, revive, tmp_path):
    path, guests, exp = revive
    b = fmc.Batch([CALF], [SEED])
    b.restart(0, path)
    b.run(1500)
    b.write_revive(0, str(tmp_path))
    st = b.state(0)
    r = fmc.read_revive(str(tmp_path / "REVIVE"), CALF)
    assert r["guests"][0].shape[0] == st["nmol0"]
    assert np.array_equal(r["guests"][0], b.guest_coords(0, 0))
    assert r["energy"][0] == st["energy0"] and r["production"] is True
    assert r["chainstats"][0] == st["prodcount"] and r["chainstats"][1] == st["N"]
    c = fmc.Chain(CALF, seed=SEED)
    c.restart(str(tmp_path / "REVIVE"))
    # the single point of the checkpointed state against the oracle's of the same coordinates
    # (the running energy differs from it by design: the reference's move loop starts its tail
    # correction at zero, so the first insertion or deletion adds the whole correction)
    orc = oracle_mod.Chain(CALF, seed=SEED)
    orc.load_guests(0, r["guests"][0].reshape(-1, 3))
    sp = c.info()["spenergy"]
    assert abs(sp - orc.scalars()["spenergy"]) <= REL * abs(sp)
    assert os.path.getsize(tmp_path / "REVCON") > 0


def test_control_restart_reads_the_branch_revive(fmc, oracle_mod, revive, tmp_path):
    """A deck whose CONTROL says `restart` continues from branch01/REVIVE beside it on both paths
    (gcmc.f:353-418): the plain chain (node 0) and both chains of a batch opened from that deck
    (node 1 of a run that left one branch reads branch01 too) follow the oracle's restarted chain."""
    from test_restart_branch import restart_deck

    path, guests, exp = revive
    work = restart_deck(tmp_path / "job")
    os.makedirs(os.path.join(work, "branch01"))
    shutil.copy(path, os.path.join(work, "branch01", "REVIVE"))
    c = fmc.Chain(work, seed=SEED)
    assert c.guest_coords(0).shape[0] == len(guests)
    _compare_traces(c.run(400), _oracle_restart(oracle_mod, guests, exp).run(400))
    b = fmc.Batch([work, work], [SEED, (1, 2, 3, 4)])
    assert b.state(0)["nmol0"] == len(guests) and b.state(1)["nmol0"] == len(guests)
    tr, _ = b.run(400, trace=True)
    _compare_traces(tr[0], _oracle_restart(oracle_mod, guests, exp).run(400))
    _compare_traces(tr[1], _oracle_restart(oracle_mod, guests, exp, seed=(1, 2, 3, 4)).run(400))
    # without a branch REVIVE the deck starts from its CONFIG, like the deck without the directive
    empty = restart_deck(tmp_path / "fresh")
    assert fmc.Chain(empty, seed=SEED).guest_coords(0).shape[0] == 0
