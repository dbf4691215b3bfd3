"""A SystemDesc built straight from the synthetic generator's arrays (no deck files)."""
import math

import numpy as np

ENGUNIT_KCAL = 418.4


def desc_from_synth(fmc, fw, gas, pressure_bar, temp, kmax, rcut=12.5, alpha=0.26, eq=-5000, prod=-5000):
    """fw: synth.Framework; gas: synth.GASES entry.  Types, pair lines and moves as
    synth.write_inputs writes them (guest sites first, Lorentz-Berthelot lj lines, equal insert /
    delete / displace / rotate weights)."""
    from fastmc_b200 import synth

    gname, sites = gas
    types, lj = [], {}
    for s, m, q, x, y, z, e, sg in sites:
        if s not in types:
            types.append(s)
            lj[s] = (e, sg)
    for t, _, _ in synth.FRAMEWORK_TYPES:
        if t in fw.names and t not in types:
            types.append(t)
            lj[t] = fw.lj[t]
    tix = {t: i + 1 for i, t in enumerate(types)}
    vdw = []
    for i, a in enumerate(types):
        for b in types[: i + 1]:
            eps = math.sqrt(lj[a][0] * lj[b][0])
            sig = 0.5 * (lj[a][1] + lj[b][1]) if eps > 0 else 0.0
            # the pair parameters at the 6 decimals the deck writer prints, so that the two routes
            # differ only by the last bit of a number's conversion
            eps, sig = float(f"{eps:.6f}"), float(f"{sig:.6f}")
            vdw.append((tix[a], tix[b], 2, (eps * ENGUNIT_KCAL, sig, 0.0, 0.0, 0.0)))
    mass = np.array([s[1] for s in sites])
    tmpl = np.array([[s[3], s[4], s[5]] for s in sites])
    tmpl = tmpl - (mass[:, None] * tmpl).sum(0) / mass.sum()
    masses = {t: m for t, m, _ in synth.FRAMEWORK_TYPES}
    L = np.diag(fw.cell)
    imcon = 1 if abs(L[0] - L[1]) <= 1e-8 * L[0] and abs(L[1] - L[2]) <= 1e-8 * L[0] else 2
    guest = {"name": gname.lower(), "mass": mass, "charge": [s[2] for s in sites], "template": tmpl,
             "type": [tix[s[0]] for s in sites], "pressure_pa": pressure_bar * 1e5,
             "move_freq": [0.25, 0.25, 0.25, 0, 0, 0, 0, 0.25, 0]}
    return fmc.SystemDesc.from_arrays(imcon, fw.cell, alpha, kmax, rcut, types, fw.xyz, fw.charges,
                                      [tix[n] for n in fw.names], [guest], vdw, temp, eq, prod,
                                      fw_mass=[masses[n] for n in fw.names], max_guest_atoms=30000)
