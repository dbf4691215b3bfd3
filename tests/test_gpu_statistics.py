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
