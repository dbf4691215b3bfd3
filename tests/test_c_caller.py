"""The drop-in ABI from a C program (tests/c_caller/dropin.c): compiled against
include/fastmc_b200.h alone and linked to the library, as a C host or a Fortran code through
bind(C) would use it.  On the host: the deck tables, the footprint, the tile list, the restart
branch choice and the error path; on the GPU: one insertion pass and its commit, equal to the same calls through Python."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import PKG, ROOT


@pytest.fixture(scope="module")
def dropin(tmp_path_factory, fmc):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    out = str(tmp_path_factory.mktemp("cc") / "dropin")
    libdir = os.path.join(PKG, "lib")
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_caller", "dropin.c"), "-L", libdir, "-lfastmc_b200",
                    f"-Wl,-rpath,{libdir}", "-o", out], check=True)
    return out


def _run(exe, *args):
    r = subprocess.run([exe, *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.mark.parametrize("name", ["small", "large", "calf20"])
def test_c_caller_host_entry_points(fmc, decks, dropin, name):
    from fastmc_b200 import placement

    got = _run(dropin, "host", decks[name])
    info = fmc.deck_inspect(decks[name])
    assert got["K"] == info["K"] and got["imcon"] == info["imcon"] and got["nerc"] == info["mxgrid"] + 1
    b, c = placement.footprint(decks[name])
    assert got["bytes"] == b and abs(got["move_cost"] - c) <= 1e-6 * c
    assert got["tiles"] == len(fmc.batch_tiles())
    br = fmc.restart_branch(decks[name], 0)
    assert got["restart_rc"] == (br["revive"] is not None) and got["prevnodes"] == br["prevnodes"]
    assert got["revive"] == (br["revive"] or "") and got["outdir"] == br["outdir"]
    assert got["missing_rc"] != 0 and got["missing_msg"] == 1


@pytest.mark.gpu
def test_c_caller_dropin_pass_equals_python(fmc, oracle_mod, decks, dropin):
    d = decks["small"]
    tmpl, _, _, _ = oracle_mod.Chain(d).guest_template(0)
    lines = open(os.path.join(d, "CONFIG")).read().split("\n")
    cell = np.array([[float(v) for v in lines[k].split()] for k in (2, 3, 4)])
    xyz = tmpl + np.array([0.31, 0.52, 0.27]) @ cell
    got = _run(dropin, "chain", d, *xyz.reshape(-1).tolist())
    c = fmc.Chain(d, seed=(12, 34, 56, 78))
    e1 = c.ewald1_guest(0, xyz, fmc.INSERT)
    e2, ev = c.guest_realspace(0, xyz, -1)
    assert got["ewld1"] == e1 and got["ewld2"] == e2 and got["vdw"] == ev
    c.commit(fmc.INSERT, 0, -1, xyz)
    x2, xv = c.guest_realspace(0, xyz, 0)
    assert got["ewld2_excl"] == x2 and got["vdw_excl"] == xv
