"""Statistical pin: CALF-20 + CO2 at 303.15 K and 0.9948 bar against the reference's own
long run (examples/restart/1_restart_example_with_completed_long_simulation_data/OUTPUT:
151-161: <N> = 91.811778 +/- 4.230, Q_st = 9.625409 +/- 0.058306 kcal/mol, 2.26e8 moves).

296 independent chains of the batched FP64 path (one per CTA slot of the GPU) start from the
empty framework, equilibrate for 1.5e6 moves each (the loading plateaus by ~1.2e6) and
produce for 1e6 moves each (2.96e8 production moves in all).  The pooled loading and heat of
adsorption must fall inside the reference's error bars combined with the pooled estimate's
own (3 sigma).  A 4e6-move run of the same set-up gave <N> = 91.44 +/- 0.16 and
Q_st = 9.632."""
import os
import shutil

import numpy as np
import pytest

from fastmc_b200 import stats

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.abspath(__file__))
REF = {"N": (91.811778, 4.230), "Qst": (9.625409, 0.058306)}


def test_calf20_loading_and_qst_inside_reference_error_bars(fmc, tmp_path):
    d = tmp_path / "calf20"
    d.mkdir()
    src = os.path.join(ROOT, "golden", "calf20")
    for f in ("FIELD", "CONFIG"):
        shutil.copy(os.path.join(src, f), d / f)
    ctl = open(os.path.join(src, "CONTROL")).read()
    ctl = ctl.replace("steps    100000000", "steps    1000000000")
    ctl = ctl.replace("equilibration    -1500000", "equilibration    1500000")
    (d / "CONTROL").write_text(ctl)
    n = 296
    seeds = [(103, 112, 53, 1 + (152 + i) % 168) for i in range(n)]
    b = fmc.Batch([str(d)] * n, seeds)
    total = 0
    while total < 2_500_000:
        b.run(250_000)
        total += 250_000
    st = [b.state(i) for i in range(n)]
    assert all(s["status"] == 0 for s in st)
    assert all(s["prodcount"] == st[0]["prodcount"] > 900_000 for s in st)
    p = stats.pooled(st, 303.15)
    for key in ("N", "Qst"):
        ref, err = REF[key]
        tol = 3.0 * np.hypot(err, p[key + "_err"])
        assert abs(p[key] - ref) < tol, (key, p[key], p[key + "_err"], ref, err)
    # the pooled estimate is far tighter than the reference's own error bar
    assert p["N_err"] < 1.0


# ---------------------------------------------------------------- windows and final report
@pytest.fixture(scope="module")
def window_decks(decks, tmp_path_factory):
    """The mixture (CO2 + N2) and single-species decks with production from the first move and
    an averaging window of 150 moves."""
    out = {}
    for name in ("mixture", "ortho1"):
        d = tmp_path_factory.mktemp("win_" + name)
        for f in ("FIELD", "CONFIG", "CONTROL"):
            shutil.copy(os.path.join(decks[name], f), d / f)
        ctl = (d / "CONTROL").read_text()
        ctl = "\n".join("equilibration 0" if ln.startswith("equilibration") else ln for ln in ctl.split("\n"))
        ctl = ctl.replace("finish", "averaging window 150\nfinish")
        (d / "CONTROL").write_text(ctl)
        out[name] = str(d)
    return out


def _close(a, b, rel=1e-9):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    scale = np.maximum(np.abs(b), 1.0)
    ok = (np.abs(a - b) <= rel * scale) | (np.isnan(a) & np.isnan(b)) | (np.isinf(a) & (a == b))
    return bool(ok.all())


def _check_windows(w, wo):
    assert w["avcount"] == wo["avcount"] > 5 and w["rollcount"] == wo["rollcount"]
    for k in ("sum", "var", "avg", "seltot"):
        assert _close(w[k], wo[k]), (k, w[k], wo[k])


@pytest.mark.parametrize("name", ["mixture", "ortho1"])
def test_plain_windows_and_final_stats_match_oracle(fmc, oracle_mod, window_decks, name, tmp_path):
    deck, seed = window_decks[name], (12, 34, 56, 78)
    c = fmc.Chain(deck, seed=seed)
    orc = oracle_mod.Chain(deck, seed=seed)
    c.run(1200)
    orc.run(1200)
    _check_windows(c.window_stats(), orc.window_stats())
    fs, fo = c.final_stats(), orc.final_stats()
    assert fs[0] == fo[0] == 1200
    assert _close(fs, fo), (fs, fo)
    # the chain's report is the host writer's on the same statistics
    c.write_report(str(tmp_path / "a"))
    fmc.write_report(deck, fs, str(tmp_path / "b"), seltot=c.window_stats()["seltot"])
    assert (tmp_path / "a").read_bytes() == (tmp_path / "b").read_bytes()
    assert "Data reported from node   0" in (tmp_path / "a").read_text()


def test_batch_windows_and_final_stats_match_oracle(fmc, oracle_mod, window_decks, tmp_path):
    decks = [window_decks["mixture"], window_decks["ortho1"], window_decks["mixture"]]
    seeds = [(12, 34, 56, 78), (1, 2, 3, 4), (5, 6, 7, 8)]
    b = fmc.Batch(decks, seeds)
    b.run(500)
    b.run(700)
    for i, (d, s) in enumerate(zip(decks, seeds)):
        orc = oracle_mod.Chain(d, seed=s)
        orc.run(1200)
        _check_windows(b.window_stats(i), orc.window_stats())
        fb, fo = b.final_stats(i), orc.final_stats()
        assert fb[0] == fo[0] == 1200
        assert _close(fb, fo), (i, fb, fo)
    b.write_report(0, str(tmp_path / "r0"))
    assert (tmp_path / "r0").read_text().count("guest  1 over guest  2") == 1
