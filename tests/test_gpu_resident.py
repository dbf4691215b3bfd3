"""The plain path's resident pass kernel: one launch serves a chain's passes from a pinned
mailbox.  Its passes must equal the one-launch passes bit for bit (same blocks, same order of
summation), it must end by itself when no pass comes and start again on the next one, and
other device work on the chain (single point, guest upload, S(k) read-back, the drop-in calls)
must stop it first.  It is off by default; these tests switch it on."""
import time

import numpy as np
import pytest

from test_gpu_plain import _compare_traces

pytestmark = pytest.mark.gpu


def _trace(fmc, deck, seed, n, resident):
    c = fmc.Chain(deck, seed=seed)
    c.resident(resident)
    tr = c.run(n, trace=True)
    return c, tr


@pytest.mark.parametrize("name", ["small", "large", "multijump", "mixture"])
def test_resident_passes_equal_launched_passes(fmc, oracle_mod, decks, name):
    seed = (12, 34, 56, 78)
    n = 3000 if name != "large" else 1500
    c_on, t_on = _trace(fmc, decks[name], seed, n, True)
    c_off, t_off = _trace(fmc, decks[name], seed, n, False)
    on, launches, served = c_on.resident()
    assert on and launches >= 1 and served > 0.9 * n
    for key in ("mtype", "randchoice", "accepted", "nmols_after", "estep", "ewld1", "ewld2", "vdw"):
        assert np.array_equal(t_on[key], t_off[key]), key
    assert np.array_equal(c_on.sk(), c_off.sk())
    _compare_traces(t_on, oracle_mod.Chain(decks[name], seed=seed).run(n))


def test_resident_kernel_ends_when_idle_and_restarts(fmc, oracle_mod, decks):
    d, seed = decks["small"], (3, 1, 4, 1)
    c = fmc.Chain(d, seed=seed)
    c.resident(True)
    parts = []
    for _ in range(4):
        parts.append(c.run(300, trace=True))
        time.sleep(0.2)  # well past the kernel's idle limit
    on, launches, served = c.resident()
    assert on and launches >= 4
    _compare_traces(np.concatenate(parts), oracle_mod.Chain(d, seed=seed).run(1200))


def test_resident_kernel_stops_for_other_device_work(fmc, oracle_mod, decks):
    """Single points, S(k) reads and drop-in passes between resident passes."""
    d, seed = decks["small"], (5, 6, 7, 8)
    c = fmc.Chain(d, seed=seed)
    c.resident(True)
    orc = oracle_mod.Chain(d, seed=seed)
    got = []
    for k in range(5):
        got.append(c.run(200, trace=True))
        sk = c.sk()
        assert np.all(np.isfinite(sk))
        c.single_point()
    ref = orc.run(1000)
    _compare_traces(np.concatenate(got), ref)
