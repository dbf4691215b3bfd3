"""Pressure equilibration (CONTROL desorb / adsorb press / adsorb guests / packing fraction /
finishment; gcmc.f:637-696, 1796-1808) in the oracle, and the decks the product refuses for it."""
import os
import shutil

import numpy as np
import pytest


def test_oracle_pressures_move_then_settle(oracle_mod, decks):
    c = oracle_mod.Chain(decks["pressure_eq"], seed=(12, 34, 56, 78))
    p0, tol = c.pressures()
    assert np.allclose(p0, [0.5e5, 0.5e5]) and tol == 1e-9
    seen = []
    for _ in range(14):
        c.run(400)
        seen.append(c.pressures()[0].copy())
    seen = np.array(seen)
    # adjusted at every 400-move check while equilibrating, the total kept
    assert len({tuple(r) for r in seen[:12]}) == 12
    assert np.allclose(seen.sum(axis=1), 1e5)
    # forced to settle once the move count passes -50 x eqsteps = 5000: the count restarts at 0
    p, tol = c.pressures()
    assert tol == 0.0 and np.array_equal(seen[-1], seen[-2])
    assert c.ints()["gcmccount"] < 5000


def _variant(src, dst, ctl_edit=None, field_edit=None):
    shutil.copytree(src, dst)
    for name, edit in (("CONTROL", ctl_edit), ("FIELD", field_edit)):
        if edit:
            p = os.path.join(dst, name)
            text = open(p).read()
            open(p, "w").write(edit(text))
    return dst


def test_pressure_equilibration_needs_desorb_1(fmc, oracle_mod, decks, tmp_path):
    d = _variant(decks["pressure_eq"], str(tmp_path / "nodesorb"), ctl_edit=lambda t: t.replace("desorb 1\n", ""))
    with pytest.raises(fmc.FastMCError) as e:
        fmc.deck_inspect(d)
    assert e.value.code == -2
    with pytest.raises(oracle_mod.OracleError):
        oracle_mod.Chain(d)


def test_deck_parses_pressure_equilibration(fmc, decks):
    info = fmc.deck_inspect(decks["pressure_eq"])
    assert info["nspecies"] == 2


def test_pressure_equilibration_needs_guests_first_in_field(fmc, decks, tmp_path):
    """The reference indexes the per-guest pressure arrays by FIELD molecule index."""
    def framework_first(text):
        lines = text.split("\n")
        i0 = lines.index("Framework")
        i1 = lines.index("finish", i0) + 1
        first = next(i for i, ln in enumerate(lines) if ln.startswith("&guest"))
        return "\n".join(lines[:first] + lines[i0:i1] + lines[first:i0] + lines[i1:])

    d = _variant(decks["pressure_eq"], str(tmp_path / "fwfirst"), field_edit=framework_first)
    with pytest.raises(fmc.FastMCError) as e:
        fmc.deck_inspect(d)
    assert e.value.code == -2 and "guests first" in str(e.value)
