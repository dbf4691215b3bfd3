"""numguests.out and his.xyz (gcmc.f:418-450, 785-792, 1937-1951, 2491-2517) as the oracle writes
them: one record per species every nnumg moves, consistent with the move trace, and the guest
geometries every |nhis| moves.  Formats: (i9,i7,2f20.6,6i4) and (i6,/,'step ',i7) + (2x,a1,3f16.6)."""
import os
import shutil

import numpy as np


def with_outputs(src, dst, nnumg, nhis):
    os.makedirs(dst, exist_ok=True)
    for f in ("FIELD", "CONFIG"):
        shutil.copy(os.path.join(src, f), os.path.join(dst, f))
    ctl = open(os.path.join(src, "CONTROL")).read()
    ctl = ctl.replace("finish", f"numguests {nnumg}\nhistory {nhis}\nfinish")
    open(os.path.join(dst, "CONTROL"), "w").write(ctl)
    return dst


def read_numguests(path):
    rows = []
    for ln in open(path):
        rows.append((int(ln[0:9]), int(ln[9:16]), float(ln[16:36]), float(ln[36:56]))
                    + tuple(int(ln[56 + 4 * k:60 + 4 * k]) for k in range(6)))
    return rows


def test_oracle_numguests_follows_the_trace(oracle_mod, decks, tmp_path):
    deck = with_outputs(decks["mixture"], str(tmp_path / "deck"), 7, -50)
    out = tmp_path / "out"
    out.mkdir()
    c = oracle_mod.Chain(deck, seed=(12, 34, 56, 78))
    c.open_outputs(str(out))
    tr = c.run(700)
    c.open_outputs(None)
    assert sorted(os.listdir(out)) == ["his01.xyz", "his02.xyz", "numguests01.out", "numguests02.out"]
    rows = [read_numguests(out / f"numguests0{g + 1}.out") for g in range(2)]
    steps = tr["step"][tr["step"] % 7 == 0]
    nmol = [0, 0]
    eng = [0.0, 0.0]
    k = 0
    for r in tr:
        nmol[r["iguest"]] = r["nmols_after"]
        eng[r["iguest"]] = r["energy_after"]
        if r["step"] % 7:
            continue
        for g in range(2):
            row = rows[g][k]
            assert row[0] == r["step"] and row[1] == nmol[g]
            assert abs(row[2] - eng[g]) <= 5e-7
            me = g == r["iguest"]
            de = r["estep"] if (me and r["accepted"] and r["mtype"] != 7) else 0.0
            assert abs(row[3] - de) <= 5e-7
            flags = [0] * 6
            if me:
                m = r["mtype"]
                flags = [int(m == 1), int(m == 2), {3: 1, 4: 2, 5: 3}.get(m, 0), {6: 1, 8: 2}.get(m, 0), 0, 0]
            assert list(row[4:]) == flags, (r, row)
        k += 1
    assert k == len(steps) == len(rows[0]) == len(rows[1])
    # his.xyz: a frame every 50 moves, the count line then "step n", one line per site
    lines = open(out / "his01.xyz").read().split("\n")
    frames = [i for i, ln in enumerate(lines) if ln.startswith("step ")]
    assert len(frames) == 700 // 50
    assert lines[frames[-1]] == "step %7d" % 700
