"""Probability plots on the host: CONTROL parsing, grid dimensions, the cube writer's format
and its atomic numbers (no GPU).  The deck is the reference's probability-plot example
(examples/advance/1_probability_plot_unary: CO2 in CALF-20, plots of site 1 and of sites 2+3,
grid spacing 0.15, grid factors 2 2 2)."""
import json
import os
import shutil

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PP = os.path.join(HERE, "golden", "probplot")


def test_plots_and_grid_dimensions_match_oracle(fmc, oracle_mod):
    info = fmc.deck_inspect(PP)
    orc = oracle_mod.Chain(PP)
    g = orc.prob()
    assert info["nplots"] == 2 == g.shape[0]
    assert info["ngrid"] == g.shape[1:]
    # gcmc.f:250-252: factor * ceiling(length / (spacing * factor))
    assert all(n % 2 == 0 for n in info["ngrid"])


def test_atomic_numbers_agree_with_reference_windows(fmc):
    """Inside and at the edges of every mass window of the reference's atmnumber."""
    wins = json.load(open(os.path.join(HERE, "golden", "atmnumber_windows.json")))
    first = {}
    for lo, hi, z in wins:
        if lo > hi:  # the reference's Ru window is written 109.9-101.5 and holds no mass
            assert fmc.atomic_number(0.5 * (lo + hi)) != z
            continue
        for m in (lo, hi, 0.5 * (lo + hi)):
            first.setdefault(m, z)  # the first window holding a mass decides, as in the if-chain
    for m, z in first.items():
        assert fmc.atomic_number(m) == z, (m, z)
    assert fmc.atomic_number(65.38) == 30 and fmc.atomic_number(15.999) == 8
    assert fmc.atomic_number(2.5) == 0


def _fortran_e(x):
    if x == 0:
        return "0.000000E+00"
    m, e = ("%.5e" % abs(x)).split("e")
    return ("-" if x < 0 else "") + "0." + m.replace(".", "") + "E%+03d" % (int(e) + 1)


def test_cube_writer_format(fmc, tmp_path):
    info = fmc.deck_inspect(PP)
    na, nb, nc = info["ngrid"]
    rng = np.random.default_rng(3)
    grid = rng.random((na, nb, nc)) * (rng.random((na, nb, nc)) < 0.01)
    path = tmp_path / "prob.cube"
    fmc.write_prob_cube(PP, str(path), grid, 1000)
    lines = open(path).read().split("\n")
    assert lines[0] == "probability cube file"
    assert lines[1] == "outer loop a, middle loop     b, inner loop c"
    nf = int(lines[2][:6])
    assert nf == info["nframework"]
    assert [int(l[:6]) for l in lines[3:6]] == [na, nb, nc]
    atoms = lines[6:6 + nf]
    assert all(len(a) == 54 for a in atoms)
    body = lines[6 + nf:]
    vals = [body_line[i:i + 15] for body_line in body for i in range(0, len(body_line), 15)]
    assert len(vals) == na * nb * nc
    # six values a line, and a line ends at every c row
    assert max(len(l) for l in body) <= 90 and all(len(l) % 15 == 0 for l in body if l)
    # the cell volume in Bohr^3 of one grid cell, as writeprob forms it
    c = np.array(info_cell(PP)) * 1.889725989
    vol = ((c[1] * c[5] - c[2] * c[4]) / (na * nb) * c[6] / nc + (c[2] * c[3] - c[0] * c[5]) / (na * nb) * c[7] / nc
           + (c[0] * c[4] - c[1] * c[3]) / (na * nb) * c[8] / nc)
    flat = grid.reshape(-1)
    for k in np.nonzero(flat)[0][:50]:
        assert vals[k].strip() == _fortran_e(flat[k] / vol / 1000)


def info_cell(deck):
    lines = open(os.path.join(deck, "CONFIG")).read().split("\n")
    return [float(v) for l in lines[2:5] for v in l.split()]
