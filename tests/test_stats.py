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


def test_report_block_matches_reference_output(tmp_path):
    """The report writer against the per-node block of the CALF-20 example's OUTPUT
    (gcmc.f:2052-2108), fed the moments, multiplier and errors that block prints."""
    import os

    import fastmc_b200

    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "calf20")
    ref = open(os.path.join(gold, "report_node0.txt")).read().split("\n")
    fs = np.zeros(15)
    fs[0] = 100000001
    fs[1:6] = [91.811777992, -756.809149592, -69669.494245516, 8449.961248488, 574495.827703705]
    fs[12], fs[13] = 0.058306353, 0.000088536
    out = tmp_path / "report"
    fastmc_b200.write_report(gold, fs, out)
    got = out.read_text().split("\n")
    assert len(got) == len(ref)
    for g, r in zip(got, ref):
        if "Isosteric heat of adsorption" in r or "Heat capacity, Cv" in r:
            # computed from the 9-decimal moments above rather than the run's own
            assert g[:65] == r[:65] and abs(float(g[65:]) - float(r[65:])) < 2e-8, (g, r)
        else:
            assert g == r


def test_report_for_a_mixture_has_each_species_and_the_selectivity(decks, tmp_path):
    """Two guest species: a block per species, then one selectivity block for the pair
    (gcmc.f:2052-2117 writes `guest j over guest i` for j < i)."""
    import fastmc_b200

    fs = np.zeros(1 + 14 * 2)
    fs[0] = 5000
    fs[1:6] = [3.0, -20.0, -65.0, 10.0, 420.0]
    fs[15:20] = [1.5, -6.0, -10.0, 2.5, 40.0]
    sel = np.array([[0.0, 0.0], [2.25, 0.0]])
    out = tmp_path / "report"
    fastmc_b200.write_report(decks["mixture"], fs, out, seltot=sel)
    text = out.read_text()
    assert text.count("Multiplier:") == 2 and text.count("Isosteric heat of adsorption") == 2
    assert "guest  1 over guest  2" in text and "guest  2 over guest  1" not in text
    line = next(ln for ln in text.split("\n") if "<S>:" in ln)
    assert abs(float(line.split()[-1]) - 2.25) < 1e-9
