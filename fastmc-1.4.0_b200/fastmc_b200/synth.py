"""Seeded synthetic GCMC inputs in FastMC's own CONTROL / FIELD / CONFIG formats.

The reference benchmarks on user frameworks; here seeded synthetic rigid frameworks stand in
for them.  Every workload below is written as real input files so the GPU path and the CPU
oracle read identical inputs through the reference's parsing rules:

* FIELD   -- readinputs.f:11-307 (guest molecule first, then the framework, then VDW pairs)
* CONFIG  -- readinputs.f:309-513 (levcfg 0, coordinates as three 20-character fields)
* CONTROL -- readinputs.f:515-914 (explicit ``ewald sum alpha k1 k2 k3``)

Workloads (sizes follow the benchmark definitions):

* ``plain_small``  : cubic cell a=25.832 A, 424 framework atoms, CO2 at 0.15 bar, kmax 8.
* ``plain_large``  : the same framework replicated 2x2x2 (3392 atoms, a=51.664 A), CO2 at 1 bar,
  kmax 12.
* ``batched``      : 16 orthorhombic frameworks (edges U(18,52) A, rho 0.025 A^-3, edges below
  2*rcut replicated) x 16 pressures log-spaced 0.01-10 bar = 256 chains, kmax per axis from a
  0.9 A^-1 reciprocal cutoff.
* ``mixture``      : the batched frameworks with a 15:85 CO2/N2 mixture at 1 bar.
* ``serving``      : a Poisson stream of isotherm-point requests (fresh frameworks of
  400-6000 atoms, CO2 / N2 / CH4, T in 273-348 K, P log-uniform 0.01-10 bar).
"""
import math
import os

import numpy as np

FRAMEWORK_TYPES = (("Zn", 65.38, 0.08), ("O", 15.9994, 0.24), ("C", 12.0107, 0.45), ("H", 1.00794, 0.23))

# guest definitions: (name, [(site, mass, charge, x, y, z, eps kcal/mol, sigma A)])
CO2 = ("CO2", [("Cx", 12.0107, 0.70, 0.0, 0.0, 0.0, 0.054, 2.80),
               ("Ox", 15.9994, -0.35, 1.16, 0.0, 0.0, 0.157, 3.05),
               ("Ox", 15.9994, -0.35, -1.16, 0.0, 0.0, 0.157, 3.05)])
N2 = ("N2", [("Nx", 14.0067, -0.482, 0.55, 0.0, 0.0, 0.072, 3.31),
             ("COM", 0.0, 0.964, 0.0, 0.0, 0.0, 0.0, 0.0),
             ("Nx", 14.0067, -0.482, -0.55, 0.0, 0.0, 0.072, 3.31)])
CH4 = ("CH4", [("CM", 16.04246, 0.0, 0.0, 0.0, 0.0, 0.294, 3.73)])
GASES = {"CO2": CO2, "N2": N2, "CH4": CH4}

RCUT = 12.5
ALPHA = 0.26


class Framework:
    """A rigid synthetic framework: cell (3x3, rows a,b,c), atoms, per-type LJ."""

    def __init__(self, cell, names, xyz, charges, lj):
        self.cell = np.asarray(cell, dtype=np.float64)
        self.names = list(names)
        self.xyz = np.asarray(xyz, dtype=np.float64)
        self.charges = np.asarray(charges, dtype=np.float64)
        self.lj = dict(lj)  # type name -> (eps, sigma)

    @property
    def natoms(self):
        return len(self.names)

    def replicate(self, na, nb, nc):
        cell = self.cell * np.array([[na], [nb], [nc]])
        shifts = [i * self.cell[0] + j * self.cell[1] + k * self.cell[2]
                  for i in range(na) for j in range(nb) for k in range(nc)]
        xyz = np.concatenate([self.xyz + s for s in shifts])
        names = self.names * len(shifts)
        q = np.tile(self.charges, len(shifts))
        return Framework(cell, names, xyz, q, self.lj)


def _place_atoms(rng, lengths, n, dmin=1.8, shift=None):
    """Uniform random positions in an orthorhombic box with a periodic minimum separation; with
    `shift`, the lattice also holds the box shifted by that vector (the half-shift cells)."""
    L = np.asarray(lengths, dtype=np.float64)
    shifts = [np.zeros(3)] + ([np.asarray(shift, dtype=np.float64)] if shift is not None else [])
    pts = np.zeros((n, 3))
    count = 0
    tries = 0
    while count < n:
        tries += 1
        if tries > 200 * n + 10000:
            raise RuntimeError("could not place atoms at the requested density")
        p = rng.uniform(0.0, 1.0, 3) * L
        if count:
            close = False
            for sv in shifts:
                d = pts[:count] - p + sv
                d -= L * np.round(d / L)
                close = close or np.min(np.einsum("ij,ij->i", d, d)) < dmin * dmin
            if close:
                continue
        pts[count] = p
        count += 1
    return pts


def make_framework(lengths, natoms, seed, shift=None):
    """Synthetic framework: type mix Zn 8% / O 24% / C 45% / H 23%, q ~ N(0, 0.4) shifted to
    sum to zero, LJ eps ~ U(0.02, 0.3) kcal/mol and sigma ~ U(2.5, 3.8) A per type."""
    rng = np.random.default_rng(seed)
    counts = [int(round(f * natoms)) for _, _, f in FRAMEWORK_TYPES]
    counts[2] += natoms - sum(counts)
    names = []
    for (name, _, _), c in zip(FRAMEWORK_TYPES, counts):
        names += [name] * c
    xyz = _place_atoms(rng, lengths, natoms, shift=shift)
    q = rng.normal(0.0, 0.4, natoms)
    q -= q.mean()
    q = np.round(q, 10)
    q[-1] -= q.sum()
    q = np.round(q, 10)
    lj = {}
    for name, _, _ in FRAMEWORK_TYPES:
        lj[name] = (float(rng.uniform(0.02, 0.3)), float(rng.uniform(2.5, 3.8)))
    cell = np.diag(np.asarray(lengths, dtype=np.float64))
    return Framework(cell, names, xyz, q, lj)


def half_shift_framework(imcon, edge, seed, rho=0.025):
    """A framework in the box of a half-shift cell: imcon 4 (truncated octahedron in an a x a x a
    box), 5 (rhombic dodecahedron, a x a x sqrt(2) a) or 7 (hexagonal prism, sqrt(3) b x b x c with
    c = b = edge).  The cell's lattice holds the box shifted by half its a, b (and c for 4, 5), so
    the periodic cell is half the box and holds rho x box volume / 2 atoms."""
    if imcon == 4:
        L = (edge, edge, edge)
        shift = (edge / 2, edge / 2, edge / 2)
    elif imcon == 5:
        L = (edge, edge, math.sqrt(2.0) * edge)
        shift = (edge / 2, edge / 2, L[2] / 2)
    elif imcon == 7:
        L = (math.sqrt(3.0) * edge, edge, edge)
        shift = (L[0] / 2, edge / 2, 0.0)
    else:
        raise ValueError("imcon must be 4, 5 or 7")
    n = int(round(rho * L[0] * L[1] * L[2] / 2))
    return make_framework(L, n, seed, shift=shift)


def slab_framework(edge, thickness, height, seed, rho=0.025):
    """A slab (imcon 6): atoms in an edge x edge x thickness layer at the bottom of an
    edge x edge x height cell, periodic in the plane only; rho atoms per A^3 of the layer."""
    n = int(round(rho * edge * edge * thickness))
    fw = make_framework((edge, edge, thickness), n, seed)
    fw.cell = np.diag([edge, edge, float(height)])
    return fw


def _fmt(x):
    return f"{x:.10f}"


def _pair_line(a, b, eps, sig, form):
    """A FIELD vdW line of the given functional form whose well matches LJ(eps, sig)."""
    r6 = sig ** 6
    rm = 2.0 ** (1.0 / 6.0) * sig
    if form == "lj" or eps == 0.0:
        body = f"lj {eps:.6f} {sig:.6f}"
    elif form == "12-6":
        body = f"12-6 {4 * eps * r6 * r6:.6f} {4 * eps * r6:.6f}"
    elif form == "nm":
        body = f"nm {eps:.6f} 12.0 6.0 {rm:.6f}"
    elif form == "buck":
        body = f"buck {eps * 1.0e7:.6f} {sig / 10.0:.6f} {4 * eps * r6:.6f}"
    elif form == "bhm":
        body = f"bhm {eps * 50.0:.6f} {12.0 / sig:.6f} {rm:.6f} {4 * eps * r6:.6f} {eps * sig ** 8:.6f}"
    elif form == "hbnd":
        body = f"hbnd {4 * eps * r6 * r6:.6f} {4 * eps * sig ** 10:.6f}"
    elif form == "snm":
        body = f"snm {eps:.6f} 12.0 6.0 {rm:.6f} 0.0"
    elif form == "mors":
        body = f"mors {eps:.6f} {rm:.6f} {6.0 / sig:.6f}"
    elif form == "wca":
        body = f"wca {eps:.6f} {sig:.6f} 0.0"
    else:
        raise ValueError(form)
    return f"{a:<8s} {b:<8s} {body}"


VDW_FORMS = ("lj", "12-6", "nm", "buck", "bhm", "hbnd", "snm", "mors", "wca")


def write_inputs(path, fw, gases, pressures_bar, temp, kmax, moves=None, eq_cycles=-5000, prod_cycles=-5000,
                 imcon=None, title="synthetic framework", rcut=RCUT, alpha=ALPHA, delr=1.0, vdw_forms=("lj",)):
    """Write CONTROL, FIELD and CONFIG for one chain into directory `path`."""
    os.makedirs(path, exist_ok=True)
    if imcon is None:
        L = np.diag(fw.cell)
        off = fw.cell - np.diag(L)
        if np.any(off != 0):
            imcon = 3
        elif abs(L[0] - L[1]) <= 1e-8 * L[0] and abs(L[1] - L[2]) <= 1e-8 * L[0]:
            imcon = 1
        else:
            imcon = 2
    moves = moves or {"insert": 0.25, "delete": 0.25, "displace": 0.25, "rotate": 0.25}
    gdefs = [GASES[g] if isinstance(g, str) else g for g in gases]
    # ---------------- FIELD
    fw_types = [t for t, _, _ in FRAMEWORK_TYPES]
    masses = {t: m for t, m, _ in FRAMEWORK_TYPES}
    lines = [title, "UNITS kcal", f"molecular types {len(gdefs) + 1}"]
    type_order = []
    lj = {}
    for gname, sites in gdefs:
        lines.append(f"&guest {gname}")
        lines.append("NUMMOLS 0")
        lines.append(f"ATOMS {len(sites)}")
        for s, m, q, x, y, z, e, sg in sites:
            lines.append(f"{s:<8s} {m:.6f} {q:.6f} {x:.6f} {y:.6f} {z:.6f}")
            if s not in type_order:
                type_order.append(s)
                lj[s] = (e, sg)
        lines.append("finish")
    lines.append("Framework")
    lines.append("NUMMOLS 1")
    lines.append(f"ATOMS {fw.natoms}")
    for name, q in zip(fw.names, fw.charges):
        lines.append(f"{name:<8s} {masses[name]:.6f} {_fmt(q)} 1 1")
    lines.append("finish")
    for t in fw_types:
        if t in fw.names and t not in type_order:
            type_order.append(t)
            lj[t] = fw.lj[t]
    pairs = []
    for i, a in enumerate(type_order):
        for b in type_order[: i + 1]:
            ea, sa = lj[a]
            eb, sb = lj[b]
            eps = math.sqrt(ea * eb)
            sig = 0.5 * (sa + sb) if eps > 0 else 0.0
            pairs.append(_pair_line(a, b, eps, sig, vdw_forms[len(pairs) % len(vdw_forms)]))
    lines.append(f"VDW {len(pairs)}")
    lines += pairs
    lines.append("close")
    with open(os.path.join(path, "FIELD"), "w") as f:
        f.write("\n".join(lines) + "\n")
    # ---------------- CONFIG
    lines = [title, f"{0:10d}{imcon:10d}{fw.natoms:10d}"]
    for row in fw.cell:
        lines.append("".join(f"{v:20.12f}" for v in row))
    for i, (name, p) in enumerate(zip(fw.names, fw.xyz)):
        lines.append(f"{name:<8s}{i + 1:10d}")
        lines.append("".join(f"{v:20.12f}" for v in p))
    with open(os.path.join(path, "CONFIG"), "w") as f:
        f.write("\n".join(lines) + "\n")
    # ---------------- CONTROL
    k1, k2, k3 = kmax
    lines = ["GCMC Run", f"temperature {temp:.6f}", f"steps {prod_cycles}", f"equilibration {eq_cycles}",
             "max guest atoms 30000", f"cutoff {rcut:.6f} angstrom", f"delr {delr:.6f} angstrom",
             f"ewald sum {alpha:.6f} {k1} {k2} {k3}"]
    for i, p in enumerate(pressures_bar):
        lines += [f"&guest {i + 1}", f"  pressure (bar) {p:.10f}", "&end"]
    for mv, fr in moves.items():
        lines.append(f"move {mv} {fr:.6f}")
    lines.append("finish")
    with open(os.path.join(path, "CONTROL"), "w") as f:
        f.write("\n".join(lines) + "\n")
    return path


# ------------------------------------------------------------------ named workloads
def plain_small_framework():
    return make_framework((25.832, 25.832, 25.832), 424, seed=0)


def write_plain_small(path, cycles=5000):
    fw = plain_small_framework()
    return write_inputs(path, fw, ["CO2"], [0.15], 298.0, (8, 8, 8), eq_cycles=-cycles, prod_cycles=-cycles,
                        title="synthetic cubic framework 424 atoms")


def write_plain_large(path, cycles=20000):
    fw = plain_small_framework().replicate(2, 2, 2)
    return write_inputs(path, fw, ["CO2"], [1.0], 298.0, (12, 12, 12), eq_cycles=-cycles, prod_cycles=-cycles,
                        title="synthetic cubic framework 3392 atoms")


def kmax_for(length, kcut=0.9):
    """Smallest kmax whose reference cutoff 1.05*2*pi*kmax/L reaches kcut."""
    return int(math.ceil(kcut * length / (2.0 * math.pi * 1.05)))


def batched_frameworks(n=16, seed=2024, rho=0.025, lo=18.0, hi=52.0, rcut=RCUT):
    """n orthorhombic frameworks; edges below 2*rcut are replicated into supercells."""
    rng = np.random.default_rng(seed)
    out = []
    for f in range(n):
        L = rng.uniform(lo, hi, 3)
        nat = max(8, int(round(rho * L.prod())))
        fw = make_framework(tuple(L), nat, seed=seed * 100 + f)
        reps = [max(1, int(math.ceil(2.0 * rcut / l - 1e-12))) for l in L]
        reps = [r if l * r > 2.0 * rcut else r + 1 for r, l in zip(reps, L)]
        if any(r > 1 for r in reps):
            fw = fw.replicate(*reps)
        out.append(fw)
    return out


def write_batched(root, n_frameworks=16, n_pressures=16, gases=("CO2",), fractions=(1.0,), total_bar=None,
                  cycles=5000, temp=298.0, seed=2024, select=None):
    """Write one input directory per chain: root/chain_FFF_PP (chain index F * n_pressures + P).
    Returns the list of dirs; with `select` (chain indices) only those chains, in that order."""
    fws = batched_frameworks(n_frameworks, seed=seed)
    dirs = []
    pressures = np.logspace(-2, 1, n_pressures)
    for f, fw in enumerate(fws):
        L = np.diag(fw.cell)
        kmax = tuple(kmax_for(l) for l in L)
        for p_i, p in enumerate(pressures):
            if select is not None and f * n_pressures + p_i not in select:
                continue
            tot = p if total_bar is None else total_bar
            parts = [tot * fr for fr in fractions]
            d = os.path.join(root, f"chain_{f:03d}_{p_i:02d}")
            write_inputs(d, fw, list(gases), parts, temp, kmax, eq_cycles=-cycles, prod_cycles=-cycles,
                         title=f"synthetic orthorhombic framework {f} ({fw.natoms} atoms)")
            dirs.append(d)
    if select is not None:
        order = {int(os.path.basename(d)[6:9]) * n_pressures + int(d[-2:]): d for d in dirs}
        return [order[i] for i in select]
    return dirs


def batched_seed(i, rank=0):
    """duni seed of chain i of the 256-chain batched workload on a rank."""
    return (12, 34, 56, (78 + 7 * i + 13 * rank) % 169)


def serving_requests(n, seed=7, rate_hz=50.0):
    """Poisson stream of isotherm-point requests: dicts with arrival time and chain inputs."""
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for i in range(n):
        t += rng.exponential(1.0 / rate_hz)
        nat = int(rng.integers(400, 6001))
        L = (nat / 0.025) ** (1.0 / 3.0)
        L = max(L, 25.2)
        gas = ["CO2", "N2", "CH4"][int(rng.integers(0, 3))]
        reqs.append({"id": i, "arrival_s": t, "natoms": nat, "edge": L, "gas": gas,
                     "temp": float(rng.uniform(273.0, 348.0)),
                     "pressure_bar": float(10 ** rng.uniform(-2, 1)),
                     "cycles": int(rng.integers(2000, 20001)), "seed": seed * 1000 + i})
    return reqs


def write_request(path, req):
    fw = make_framework((req["edge"],) * 3, req["natoms"], seed=req["seed"])
    kmax = (kmax_for(req["edge"]),) * 3
    return write_inputs(path, fw, [req["gas"]], [req["pressure_bar"]], req["temp"], kmax,
                        eq_cycles=-req["cycles"] // 2, prod_cycles=-req["cycles"] // 2,
                        title=f"serving request {req['id']}")
