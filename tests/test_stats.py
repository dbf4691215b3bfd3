"""Host observables (Q_st, Cv) against the reference's own final report of the CALF-20 run
(examples/restart/1_restart_example_with_completed_long_simulation_data/OUTPUT:151-161)."""
import numpy as np

from fastmc_b200 import stats


def test_qst_cv_reproduce_reference_report():
    # <N>, <E>, <E*N>, <N*N>, <E*E> as printed by the reference at T = 303.15 K
    N, E, EN, N2, E2 = 91.811777992, -756.809149592, -69669.494245516, 8449.961248488, 574495.827703705
    q = stats.qst(N, E, EN, N2, 303.15)
    c = stats.cv(N, E, EN, N2, E2, 303.15)
    # the printed moments carry 9 decimals; Q_st and Cv are printed as 9.625408877 and 0.006676699
    assert abs(q - 9.625408877) < 2e-5
    assert abs(c - 0.006676699) < 2e-5


def test_pooled_jackknife_of_identical_chains_is_exact():
    st = [{"N": 10.0 + (i % 2), "E": -50.0 - 3 * (i % 2), "EN": -520.0, "N2": 110.0, "E2": 2600.0} for i in range(8)]
    p = stats.pooled(st, 300.0)
    assert p["chains"] == 8 and abs(p["N"] - 10.5) < 1e-12
    assert p["N_err"] > 0 and np.isfinite(p["Qst_err"])
