"""B200-native GCMC trial-move energy path of FastMC 1.4.0.

Host-side mirror of the reference's operator interface: a `Chain` opened from a FastMC input
directory (CONTROL / FIELD / CONFIG) exposes the reference's energy routines (ewald1,
ewald1_guest, guest real space = guestlistgen + ewald2 + srfrce, single_point) and its move
loop, all evaluated on the GPU through libfastmc_b200.so.
"""
import ctypes
import os

# The server builds request slots on up to 8 worker streams beside its launch and admission
# streams.  With CUDA's default of 8 hardware work queues, streams share queues and a slot
# build can wait behind a whole batched launch queued on the same one.  32 queues (the maximum)
# keep the streams apart; the setting takes effect only if no CUDA context exists yet.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import numpy as np

from . import _lib
from ._lib import (DELETE, DISPLACE, INSERT, JUMP, MOVE_DTYPE, MULTIJUMP, NOOP, ROTATE, TRANSLATE, FastMCError, check,
                   dp, ip, lib)

__all__ = ["Chain", "SystemDesc", "Batch", "Server", "deck_inspect", "deck_voxels", "batch_tiles", "autotune_tiles", "FastMCError", "INSERT", "DELETE", "DISPLACE", "TRANSLATE", "ROTATE",
           "MOVE_DTYPE"]

_INFO_INTS = ["imcon", "kmax1", "kmax2", "kmax3", "K", "natoms", "nspecies", "ntypes", "mxgrid", "nframework",
              "moves", "nvoxels", "guest_capacity", "voxel_entries", "r14", "r15"]
_INFO_DBLS = ["alpha", "rcut", "delr", "volm", "engunit", "temp", "beta", "drewd", "dlrpot", "spenergy", "dlpeng",
              "ewald1sum", "elrc", "energy", "statvolm", "r15"]


def _voxel_lists(call):
    """(nvox, off, atoms) from a two-call voxel-list entry (sizes first, then the arrays)."""
    nvox = np.zeros(3, dtype=np.int32)
    n = ctypes.c_longlong(0)
    check(call(nvox, None, None, 0, n))
    off = np.zeros(int(np.prod(nvox)) + 1, dtype=np.int32)
    atoms = np.zeros(max(n.value, 1), dtype=np.int32)
    check(call(nvox, off, atoms, atoms.size, n))
    return tuple(int(v) for v in nvox), off, atoms[:n.value]


def deck_voxels(directory, voxel_edge=2.0):
    """The neighbour lists of a deck's framework built on the host by testing every atom against
    every voxel centre: (nvox, CSR offsets, atom indices)."""
    d = str(directory).encode()
    return _voxel_lists(lambda nv, off, at, cap, n: lib().fmc_deck_voxels(
        d, float(voxel_edge), ip(nv), None if off is None else ip(off), None if at is None else ip(at), int(cap),
        ctypes.byref(n)))


def deck_inspect(directory):
    """Parse a deck and build its tables on the host (no GPU).  Returns a dict."""
    ints = np.zeros(16, dtype=np.int32)
    dbls = np.zeros(16)
    K, nerc = ctypes.c_int(0), ctypes.c_int(0)
    d = str(directory).encode()
    check(lib().fmc_deck_inspect(d, ip(ints), dp(dbls), None, None, None, None, ctypes.byref(K), ctypes.byref(nerc)))
    info = dict(zip(_INFO_INTS[:12], ints.tolist()))
    info.update(zip(_INFO_DBLS, dbls.tolist()))
    info.update(nplots=int(ints[12]), ngrid=(int(ints[13]), int(ints[14]), int(ints[15])))
    lmn = np.zeros((K.value, 3), dtype=np.int32)
    akk = np.zeros(K.value)
    erc = np.zeros(nerc.value)
    q = np.zeros(max(info["nframework"], 1))
    check(lib().fmc_deck_inspect(d, None, None, ip(lmn), dp(akk), dp(erc), dp(q), ctypes.byref(K),
                                 ctypes.byref(nerc)))
    info.update(lmn=lmn, akk=akk, erc=erc, charges=q[: info["nframework"]])
    return info


def deck_vdw(directory):
    """The deck's vdW tables (host, no GPU): list of arrays, table 1 first."""
    n = ctypes.c_int(0)
    d = str(directory).encode()
    check(lib().fmc_deck_vdw(d, 0, None, ctypes.byref(n)))
    npts = deck_inspect(directory)["mxgrid"] + 1
    out = []
    for k in range(1, n.value + 1):
        a = np.zeros(npts)
        check(lib().fmc_deck_vdw(d, k, dp(a), None))
        out.append(a)
    return out


def atomic_number(mass):
    """Atomic number the probability cube files give a framework mass."""
    return int(lib().fmc_atomic_number(float(mass)))


def write_prob_cube(deck_dir, path, grid, steps):
    """Write one plot's grid (na, nb, nc) as a cube file, as the reference's writeprob does."""
    g = np.ascontiguousarray(grid, dtype=np.float64)
    check(lib().fmc_write_prob_cube(str(deck_dir).encode(), str(path).encode(), dp(g), int(steps)))


def write_report(deck_dir, final_stats, path, seltot=None):
    """The reference's per-node report block (gcmc.f:2052-2117) from final statistics in the
    chainstats layout ([0] production moves, 14 values a species); host only."""
    fs = np.ascontiguousarray(final_stats, dtype=np.float64)
    sel = None if seltot is None else np.ascontiguousarray(seltot, dtype=np.float64)
    check(lib().fmc_write_report(str(deck_dir).encode(), dp(fs), None if sel is None else dp(sel),
                                 str(path).encode()))


def _window(out, ng):
    o = out[2:]
    return {"avcount": int(out[0]), "rollcount": int(out[1]), "sum": o[:8 * ng].reshape(ng, 8),
            "var": o[8 * ng:16 * ng].reshape(ng, 8), "avg": o[16 * ng:24 * ng].reshape(ng, 8),
            "seltot": o[24 * ng:24 * ng + ng * ng].reshape(ng, ng)}


def _prob(call):
    dims = np.zeros(4, dtype=np.int32)
    check(call(0, ip(dims), None))
    n, na, nb, nc = (int(v) for v in dims)
    out = np.zeros((n, na, nb, nc))
    for k in range(n):
        buf = np.zeros(max(na * nb * nc, 1))
        check(call(k, None, dp(buf)))
        out[k] = buf[: na * nb * nc].reshape(na, nb, nc)
    return out


class SystemDesc:
    """A system handed over as arrays (fmc_system_desc): what the reference's module arrays hold
    once its readers have run.  `from_deck` reads a deck directory into one (arrays owned by the
    library); `from_arrays` builds one from the caller's own arrays (kept alive here)."""

    def __init__(self):
        self.s = _lib.SystemDescStruct()
        self._keep = []
        self._owned = False

    @classmethod
    def from_deck(cls, directory):
        d = cls()
        check(lib().fmc_deck_describe(str(directory).encode(), ctypes.byref(d.s)))
        d._owned = True
        return d

    @classmethod
    def from_arrays(cls, imcon, cell, alpha, kmax, rcut, types, fw_xyz, fw_charge, fw_type, guests, vdw, temperature,
                    eq_steps, prod_steps, delr=1.0, engunit=418.4, fw_mass=None, max_guest_atoms=0,
                    averaging_window=0, rota_ratio=0.5):
        """types: names; fw_type and guest types 1-based.  guests: dicts with name, mass, charge,
        template (nsite, 3, centred on the mass centre), type, pressure_pa, move_freq (9), and
        optionally xyz (nmol, nsite, 3), disp_ratio, tran_ratio.  vdw: (type_i, type_j, form,
        prm[5]) with energies in internal units (10 J/mol)."""
        d = cls()
        s = d.s
        s.imcon = int(imcon)
        s.cell[:] = [float(v) for v in np.asarray(cell, dtype=np.float64).reshape(-1)]
        s.alpha = float(alpha)
        s.kmax[:] = [int(k) for k in kmax]
        s.rcut, s.rvdw, s.delr, s.engunit = float(rcut), 0.0, float(delr), float(engunit)
        names = (ctypes.c_char_p * len(types))(*[t.encode() for t in types])
        s.ntypes, s.type_names = len(types), names
        arr = lambda a, t=np.float64: d.keep(np.ascontiguousarray(a, dtype=t))  # noqa: E731
        fx, fq, ft = arr(np.asarray(fw_xyz).reshape(-1)), arr(fw_charge), arr(fw_type, np.int32)
        s.nframework = len(fq)
        s.fw_xyz, s.fw_charge, s.fw_type = dp(fx), dp(fq), ip(ft)
        if fw_mass is not None:
            s.fw_mass = dp(arr(fw_mass))
        gd = (_lib.GuestDesc * len(guests))()
        for g, G in zip(gd, guests):
            t = np.asarray(G["template"], dtype=np.float64).reshape(-1, 3)
            g.name = d.keep(G.get("name", "guest").encode())
            g.nsite = len(t)
            g.mass, g.charge = dp(arr(G["mass"])), dp(arr(G["charge"]))
            g.tx, g.ty, g.tz = dp(arr(t[:, 0])), dp(arr(t[:, 1])), dp(arr(t[:, 2]))
            g.type = ip(arr(G["type"], np.int32))
            xyz = G.get("xyz")
            g.nmols = 0 if xyz is None else int(np.asarray(xyz).shape[0])
            if g.nmols:
                g.xyz = dp(arr(np.asarray(xyz).reshape(-1)))
            g.pressure_pa = float(G["pressure_pa"])
            g.move_freq[:] = [float(v) for v in G["move_freq"]]
            g.disp_ratio, g.tran_ratio = float(G.get("disp_ratio", 0.5)), float(G.get("tran_ratio", 0.5))
        s.nguest, s.guests = len(guests), gd
        vd = (_lib.VdwDesc * max(len(vdw), 1))()
        for v, (i, j, form, prm) in zip(vd, vdw):
            v.type_i, v.type_j, v.form = int(i), int(j), int(form)
            v.prm[:] = [float(x) for x in prm]
        s.nvdw, s.vdw = len(vdw), vd
        s.temperature, s.eq_steps, s.prod_steps = float(temperature), int(eq_steps), int(prod_steps)
        s.max_guest_atoms, s.averaging_window, s.rota_ratio = int(max_guest_atoms), int(averaging_window), rota_ratio
        d._keep += [names, gd, vd]
        return d

    def keep(self, obj):
        self._keep.append(obj)
        return obj

    def set_guests(self, g, xyz):
        """Replace the molecules of species g present at creation: xyz (nmol, nsite, 3)."""
        a = self.keep(np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1))
        self.s.guests[g].nmols = int(np.asarray(xyz).shape[0])
        self.s.guests[g].xyz = dp(a) if len(a) else ctypes.POINTER(ctypes.c_double)()

    def free(self):
        if self._owned:
            lib().fmc_desc_free(ctypes.byref(self.s))
            self._owned = False

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Chain:
    """One GCMC chain on one GPU (the plain FP64 path), opened from a deck directory or created
    from a SystemDesc."""

    def __init__(self, directory, seed=(12, 34, 56, 78), device=0, node=0):
        """node: this chain's node index (0-based) in a job run from one deck directory; only a
        CONTROL `restart` reads it, to pick the branch REVIVE to continue from (restart_branch)."""
        self.h = ctypes.c_void_p()
        s = np.asarray(seed, dtype=np.int32)
        if isinstance(directory, SystemDesc):
            check(lib().fmc_chain_create(ctypes.byref(directory.s), ip(s), int(device), ctypes.byref(self.h)))
        else:
            check(lib().fmc_chain_open_node(str(directory).encode(), ip(s), int(device), int(node),
                                            ctypes.byref(self.h)))

    def close(self):
        if self.h:
            lib().fmc_chain_close(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        ints = np.zeros(16, dtype=np.int32)
        dbls = np.zeros(16)
        check(lib().fmc_chain_info(self.h, ip(ints), dp(dbls)))
        out = dict(zip(_INFO_INTS, ints.tolist()))
        out.update(zip(_INFO_DBLS, dbls.tolist()))
        return out

    # ---- reference energy routines
    def ewald1(self):
        e, k = ctypes.c_double(0), ctypes.c_int(0)
        check(lib().fmc_ewald1(self.h, ctypes.byref(e), ctypes.byref(k)))
        return e.value

    def ewald1_guest(self, iguest, xyz, move, pass_=1):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        e = ctypes.c_double(0)
        check(lib().fmc_ewald1_guest(self.h, int(iguest), xyz.shape[0], dp(xyz), int(move), int(pass_),
                                     ctypes.byref(e)))
        return e.value

    def guest_realspace(self, iguest, xyz, mol=-1):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        e2, ev = ctypes.c_double(0), ctypes.c_double(0)
        check(lib().fmc_guest_realspace(self.h, int(iguest), xyz.shape[0], dp(xyz), int(mol), ctypes.byref(e2),
                                        ctypes.byref(ev)))
        return e2.value, ev.value

    def ewald1_guest_xyz(self, iguest, x, y, z, move, pass_=1):
        """ewald1_guest on separate coordinate arrays (the reference's newx/newy/newz)."""
        x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
        e = ctypes.c_double(0)
        check(lib().fmc_ewald1_guest_xyz(self.h, int(iguest), len(x), dp(x), dp(y), dp(z), int(move), int(pass_),
                                         ctypes.byref(e)))
        return e.value

    def guest_realspace_xyz(self, iguest, x, y, z, mol=-1):
        x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
        e2, ev = ctypes.c_double(0), ctypes.c_double(0)
        check(lib().fmc_guest_realspace_xyz(self.h, int(iguest), len(x), dp(x), dp(y), dp(z), int(mol),
                                            ctypes.byref(e2), ctypes.byref(ev)))
        return e2.value, ev.value

    def commit_xyz(self, move, iguest, mol, x=None, y=None, z=None):
        a = [None if v is None else np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z)]
        check(lib().fmc_commit_xyz(self.h, int(move), int(iguest), int(mol), *[None if v is None else dp(v) for v in a]))

    def commit(self, move, iguest, mol, xyz=None):
        x = None if xyz is None else np.ascontiguousarray(xyz, dtype=np.float64)
        check(lib().fmc_commit(self.h, int(move), int(iguest), int(mol), None if x is None else dp(x)))

    def reject(self):
        check(lib().fmc_reject(self.h))

    def set_guests(self, iguest, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        nsite = xyz.shape[1] if xyz.ndim == 3 else None
        nmol = xyz.shape[0] if xyz.ndim == 3 else 0
        if nsite is None:
            raise ValueError("xyz must be (nmol, nsite, 3)")
        check(lib().fmc_set_guests(self.h, int(iguest), nmol, dp(xyz)))

    def single_point(self):
        a, b = ctypes.c_double(0), ctypes.c_double(0)
        check(lib().fmc_single_point(self.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def resident(self, enable=None):
        """Passes through the resident kernel: enable True / False switches it, None only reports.
        Returns (on, launches of the kernel, passes it served)."""
        a, b = ctypes.c_longlong(0), ctypes.c_longlong(0)
        rc = lib().fmc_chain_resident(self.h, -1 if enable is None else int(bool(enable)), ctypes.byref(a),
                                      ctypes.byref(b))
        if rc < 0:
            check(rc)
        return bool(rc), a.value, b.value

    def sk(self, pending=False):
        K = self.info()["K"]
        re, im = np.zeros(K), np.zeros(K)
        check(lib().fmc_get_sk(self.h, int(bool(pending)), dp(re), dp(im)))
        return re + 1j * im

    def kvectors(self):
        K = self.info()["K"]
        lmn = np.zeros((K, 3), dtype=np.int32)
        akk = np.zeros(K)
        check(lib().fmc_kvectors(self.h, ip(lmn), dp(akk)))
        return lmn, akk

    # ---- move loop
    def run(self, nmoves, trace=True):
        rec = np.zeros(nmoves, dtype=MOVE_DTYPE) if trace else None
        check(lib().fmc_run(self.h, int(nmoves), rec.ctypes.data if trace else None))
        return rec

    def run_timed(self, nmoves, trace=False):
        """Runs nmoves; returns (trace or None, device milliseconds from CUDA events)."""
        rec = np.zeros(nmoves, dtype=MOVE_DTYPE) if trace else None
        ms = ctypes.c_float(0)
        check(lib().fmc_run_timed(self.h, int(nmoves), rec.ctypes.data if trace else None, ctypes.byref(ms)))
        return rec, float(ms.value)

    def profile(self, enable=1):
        out = np.zeros(6)
        check(lib().fmc_chain_profile(self.h, int(enable), dp(out)))
        return dict(zip(["passes", "commits", "timed_passes", "pass_ms", "K", "voxel_mean"], out.tolist()))

    def guest_coords(self, iguest=0):
        """Coordinates of species `iguest` as (nmol, nsite, 3), molecule order of the reference."""
        n, ns = ctypes.c_int(0), ctypes.c_int(0)
        check(lib().fmc_guest_coords(self.h, int(iguest), None, ctypes.byref(n), ctypes.byref(ns)))
        buf = np.zeros((max(n.value, 1), ns.value, 3))
        check(lib().fmc_guest_coords(self.h, int(iguest), dp(buf), ctypes.byref(n), ctypes.byref(ns)))
        return buf[: n.value]

    def pressures(self):
        """(partial pressures in Pa, pressure-equilibration tolerance still in force)."""
        ng = self.info()["nspecies"]
        out = np.zeros(ng + 1)
        check(lib().fmc_chain_pressures(self.h, dp(out)))
        return out[:ng], float(out[ng])

    def open_outputs(self, directory):
        """Write numguests.out and his.xyz into `directory` as the chain runs; None closes them."""
        check(lib().fmc_chain_open_outputs(self.h, None if directory is None else str(directory).encode()))

    def window_stats(self):
        ng = self.info()["nspecies"]
        out = np.zeros(2 + 24 * ng + ng * ng)
        check(lib().fmc_chain_window_stats(self.h, dp(out)))
        return _window(out, ng)

    def final_stats(self):
        """The report's statistics (averages and errors, chainstats layout)."""
        ng = self.info()["nspecies"]
        out = np.zeros(1 + 14 * ng)
        check(lib().fmc_chain_final_stats(self.h, dp(out)))
        return out

    def write_report(self, path):
        check(lib().fmc_chain_write_report(self.h, str(path).encode()))

    def prob(self):
        """Probability plots: array [plots, na, nb, nc] of binned weights (storeprob)."""
        return _prob(lambda k, dims, out: lib().fmc_chain_prob(self.h, k, dims, out))

    def write_prob(self, outdir):
        check(lib().fmc_chain_write_prob(self.h, str(outdir).encode()))

    def write_revive(self, outdir):
        """REVIVE + REVCON of the chain's state in outdir (revive, utility_pack.f:1772-1817)."""
        check(lib().fmc_chain_write_revive(self.h, str(outdir).encode()))

    def restart(self, revive_path):
        """Load a REVIVE: guests, fresh single point, production flag and statistics."""
        check(lib().fmc_chain_restart(self.h, str(revive_path).encode()))

    def stats(self, iguest=0):
        out = np.zeros(6)
        check(lib().fmc_stats(self.h, int(iguest), dp(out)))
        return dict(zip(["N", "E", "EN", "N2", "E2", "prodcount"], out.tolist()))


def _chain_args(directories, seeds):
    dirs = [str(d).encode() for d in directories]
    n = len(dirs)
    if seeds is None:
        seeds = [(12, 34, 56, (78 + i) % 169) for i in range(n)]
    s = np.ascontiguousarray(np.asarray(seeds, dtype=np.int32).reshape(n, 4))
    return (ctypes.c_char_p * n)(*dirs), s, n


def autotune_voxel_edge(directories, seeds=None, device=0, edges=(2.0, 1.5, 1.2, 1.0), moves=500):
    """The voxel edge (A) under which these chains run fastest, timed on throwaway batches;
    returns (best edge, {edge: device ms of one `moves`-move launch})."""
    arr, s, n = _chain_args(directories, seeds)
    e = np.ascontiguousarray(np.asarray(edges, dtype=np.float64))
    ms = (ctypes.c_float * len(e))()
    best = ctypes.c_double(0.0)
    check(lib().fmc_batch_autotune(n, arr, ip(s), int(device), dp(e), len(e), int(moves), ctypes.byref(best), ms))
    return best.value, {float(k): float(v) for k, v in zip(e, ms)}


def batch_tiles():
    """The batched kernel's tile shapes: a list of (threads per chain, k-vectors per thread per
    trip, candidates per trip); index 0 is the default."""
    n = lib().fmc_batch_tiles(None, None, None, 0)
    t, k, c = (np.zeros(n, dtype=np.int32) for _ in range(3))
    lib().fmc_batch_tiles(ip(t), ip(k), ip(c), n)
    return [(int(a), int(b), int(d)) for a, b, d in zip(t, k, c)]


def autotune_tiles(directories, seeds=None, device=0, voxel_edge=2.0, tiles=None, warm_moves=1000, moves=500):
    """The tile under which these chains run fastest, timed on one throwaway batch (each tile
    launched twice in palindromic order); returns (best tile index, {tile index: mean ms})."""
    arr, s, n = _chain_args(directories, seeds)
    t = np.ascontiguousarray(np.asarray(tiles if tiles is not None else range(len(batch_tiles())), dtype=np.int32))
    ms = (ctypes.c_float * len(t))()
    best = ctypes.c_int(0)
    check(lib().fmc_batch_autotune_tiles(n, arr, ip(s), int(device), float(voxel_edge), ip(t), len(t),
                                         int(warm_moves), int(moves), ctypes.byref(best), ms))
    return best.value, {int(k): float(v) for k, v in zip(t, ms)}


class Batch:
    """Many independent chains advanced by one persistent kernel (the batched path)."""

    def __init__(self, directories, seeds=None, device=0, voxel_edge=None):
        """voxel_edge: edge (A) of the neighbour-list voxels (None: the library's 2 A; see
        autotune_voxel_edge)."""
        arr, s, n = _chain_args(directories, seeds)
        self.n = n
        self.dirs = [str(d) for d in directories]
        self.h = ctypes.c_void_p()
        if voxel_edge is None:
            check(lib().fmc_batch_open(n, arr, ip(s), int(device), ctypes.byref(self.h)))
        else:
            check(lib().fmc_batch_open_edge(n, arr, ip(s), int(device), float(voxel_edge), ctypes.byref(self.h)))

    def close(self):
        if self.h:
            lib().fmc_batch_close(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, moves, trace=False):
        """Advance every chain by `moves`; returns (trace[n, moves] or None, device ms).

        A chain whose deck's equilibration + production budget runs out stops after that move
        (state()["finished"]); its remaining trace records stay zero."""
        rec = np.zeros((self.n, moves), dtype=MOVE_DTYPE) if trace else None
        ms = ctypes.c_float(0)
        check(lib().fmc_batch_run(self.h, int(moves), rec.ctypes.data if trace else None, ctypes.byref(ms)))
        return rec, float(ms.value)

    _STATE = ["status", "moves", "gcmccount", "nmol0", "nmol1", "nmol2", "nmol3", "energy0", "energy1", "energy2",
              "energy3", "elrc", "accept_ins", "accept_del", "ins_count", "del_count", "prodcount", "N", "E", "EN",
              "N2", "E2", "system", "K", "nframework", "temp", "press0", "cyc_begin", "cyc_phase", "cyc_sums",
              "cyc_end", "cyc_commit", "cyc_t0_kspace", "cyc_t0_real", "cyc_select", "cyc_trial", "finished"]

    def profile(self, enable=True):
        check(lib().fmc_batch_profile(self.h, int(bool(enable))))

    def state(self, chain):
        out = np.zeros(40)
        check(lib().fmc_batch_chain_state(self.h, int(chain), dp(out)))
        return dict(zip(self._STATE, out.tolist()))

    def timing(self):
        """Per chain of the last run: CTA start and end on the device clock (ns) and the SM it
        ran on, as an (n, 3) int64 array."""
        out = np.zeros((self.n, 3), dtype=np.int64)
        for c in range(self.n):
            check(lib().fmc_batch_chain_timing(self.h, c, out[c].ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))))
        return out

    @property
    def tile(self):
        """Index into batch_tiles() of the kernel this batch launches."""
        return int(lib().fmc_batch_get_tile(self.h))

    @tile.setter
    def tile(self, index):
        check(lib().fmc_batch_set_tile(self.h, int(index)))

    def voxels(self, chain):
        """The device-built neighbour lists of a chain's system: (nvox, CSR offsets, atom indices)."""
        return _voxel_lists(lambda nv, off, at, cap, n: lib().fmc_batch_voxels(
            self.h, int(chain), ip(nv), None if off is None else ip(off), None if at is None else ip(at), int(cap),
            ctypes.byref(n)))

    def pressures(self, chain):
        ng = self._ng(chain)
        out = np.zeros(ng + 1)
        check(lib().fmc_batch_pressures(self.h, int(chain), dp(out)))
        return out[:ng], float(out[ng])

    def write_numguests(self, chain, trace, directory, append=False):
        """numguests.out of one chain from the trace of the last run(trace=True)."""
        rec = np.ascontiguousarray(trace[chain] if trace.ndim == 2 else trace)
        check(lib().fmc_batch_write_numguests(self.h, int(chain), rec.ctypes.data, int(rec.shape[0]),
                                              str(directory).encode(), int(bool(append))))

    def window_stats(self, chain):
        ng = self._ng(chain)
        out = np.zeros(2 + 24 * ng + ng * ng)
        check(lib().fmc_batch_window_stats(self.h, int(chain), dp(out)))
        return _window(out, ng)

    def final_stats(self, chain):
        out = np.zeros(1 + 14 * self._ng(chain))
        check(lib().fmc_batch_final_stats(self.h, int(chain), dp(out)))
        return out

    def write_report(self, chain, path):
        check(lib().fmc_batch_write_report(self.h, int(chain), str(path).encode()))

    def _ng(self, chain):
        return int(deck_inspect(self.dirs[chain])["nspecies"])

    def prob(self, chain):
        return _prob(lambda k, dims, out: lib().fmc_batch_prob(self.h, int(chain), k, dims, out))

    def write_prob(self, chain, outdir):
        check(lib().fmc_batch_write_prob(self.h, int(chain), str(outdir).encode()))

    def write_revive(self, chain, outdir):
        check(lib().fmc_batch_write_revive(self.h, int(chain), str(outdir).encode()))

    def restart(self, chain, revive_path):
        """Restart chain `chain` from a REVIVE (before its first run, like the reference)."""
        check(lib().fmc_batch_restart(self.h, int(chain), str(revive_path).encode()))

    def guest_coords(self, chain, iguest=0):
        n, ns = ctypes.c_int(0), ctypes.c_int(0)
        check(lib().fmc_batch_guest_coords(self.h, int(chain), int(iguest), None, ctypes.byref(n), ctypes.byref(ns)))
        buf = np.zeros((max(n.value, 1), ns.value, 3))
        check(lib().fmc_batch_guest_coords(self.h, int(chain), int(iguest), dp(buf), ctypes.byref(n),
                                           ctypes.byref(ns)))
        return buf[: n.value]


class Server:
    """Continuous-batching server of isotherm-point requests on one GPU."""

    QUEUED, RUNNING, DONE, REJECTED, CANCELLED = 0, 1, 2, -1, -2
    _OUT = ["moves", "status", "nmol0", "nmol1", "nmol2", "nmol3", "energy0", "energy1", "energy2", "energy3",
            "prodcount", "N", "E", "EN", "N2", "E2", "accept_ins", "accept_del", "_r18", "K", "nframework",
            "temp", "press0", "budget", "finished", "N_1", "E_1", "EN_1", "N2_1", "E2_1", "gcmccount", "_"]

    def __init__(self, slots=296, device=0, mem_budget=0, k_capacity=2400, voxel_edge=2.0):
        """voxel_edge: neighbour-list voxel edge (A) of the request slots."""
        self.h = ctypes.c_void_p()
        check(lib().fmc_server_open(int(slots), int(device), int(mem_budget), int(k_capacity), ctypes.byref(self.h)))
        check(lib().fmc_server_set_voxel_edge(self.h, float(voxel_edge)))

    def close(self):
        if self.h:
            lib().fmc_server_close(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, directory, seed, moves=0):
        """Queue one request; moves=0 runs the deck's own equilibration + production cycles."""
        rid = ctypes.c_int(0)
        s = np.asarray(seed, dtype=np.int32)
        check(lib().fmc_server_submit(self.h, str(directory).encode(), ip(s), int(moves), ctypes.byref(rid)))
        return rid.value

    def cancel(self, rid):
        check(lib().fmc_server_cancel(self.h, int(rid)))

    def keep_final_state(self, enable=True):
        """Keep the guests of requests that finish from now on, for write_revive."""
        check(lib().fmc_server_keep_final_state(self.h, int(bool(enable))))

    def write_revive(self, rid, directory):
        """REVIVE + REVCON of finished request `rid` (its final state kept) into `directory`."""
        check(lib().fmc_server_write_revive(self.h, int(rid), str(directory).encode()))

    def busy(self):
        """True while a launch is in flight, a request runs or one is queued."""
        b = ctypes.c_int(0)
        check(lib().fmc_server_busy(self.h, ctypes.byref(b)))
        return bool(b.value)

    def poll_done(self, cap=4096):
        """Requests that reached a final state since the last call: list of (id, state, result)."""
        ids = np.zeros(cap, dtype=np.int32)
        states = np.zeros(cap, dtype=np.int32)
        res = np.zeros((cap, 32))
        n = ctypes.c_int(0)
        check(lib().fmc_server_poll_done(self.h, ip(ids), ip(states), dp(res), int(cap), ctypes.byref(n)))
        return [(int(ids[k]), int(states[k]), dict(zip(self._OUT, res[k].tolist()))) for k in range(n.value)]

    def step(self, moves):
        """One pipelined continuous-batching step (queues the next launch, completes the previous
        one); returns (active in the completed launch, queued, its device ms)."""
        a, q, ms = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_float(0)
        check(lib().fmc_server_step(self.h, int(moves), ctypes.byref(a), ctypes.byref(q), ctypes.byref(ms)))
        return a.value, q.value, float(ms.value)

    def poll(self, rid):
        st = ctypes.c_int(0)
        out = np.zeros(32)
        check(lib().fmc_server_poll(self.h, int(rid), ctypes.byref(st), dp(out)))
        res = dict(zip(self._OUT, out.tolist()))
        res["state"] = st.value
        if st.value == self.REJECTED:
            res["error"] = lib().fmc_last_error().decode()
        return res

    def stats(self):
        out = np.zeros(14)
        check(lib().fmc_server_stats(self.h, dp(out)))
        return dict(zip(["admitted", "retired", "launches", "admit_ms", "launch_ms", "prep_wait_ms", "prep_ms",
                         "workers", "moves", "last_moves", "prep_host_ms", "prep_device_ms", "admit_prebuilt",
                         "admit_built"], out.tolist()))

    def memory(self):
        u, b = ctypes.c_longlong(0), ctypes.c_longlong(0)
        check(lib().fmc_server_memory(self.h, ctypes.byref(u), ctypes.byref(b)))
        return u.value, b.value


# ------------------------------------------------------------------ checkpoint / restart
def write_revive_state(deck_dir, outdir, guests, production=False, chainstats=None, energy=None, eng=0.0):
    """Write outdir/REVIVE and outdir/REVCON (the reference's formats) for a deck and a host
    state: `guests` is one (nmol, nsite, 3) array per guest species."""
    gs = [np.asarray(g, dtype=np.float64).reshape(-1, 3) for g in guests]
    info = deck_inspect(deck_dir)
    ng = info["nspecies"]
    nmol = np.zeros(max(ng, 1), dtype=np.int32)
    for i in range(ng):
        ns = _species_sites(deck_dir, i)
        nmol[i] = len(gs[i]) // ns if ns else 0
    xyz = np.ascontiguousarray(np.concatenate([g.reshape(-1) for g in gs]) if gs else np.zeros(1))
    cs = np.ascontiguousarray(chainstats if chainstats is not None else np.zeros(1 + 14 * ng), dtype=np.float64)
    en = np.ascontiguousarray(energy if energy is not None else np.zeros(ng), dtype=np.float64)
    check(lib().fmc_revive_write_state(str(deck_dir).encode(), str(outdir).encode(), int(bool(production)), ip(nmol),
                                       dp(xyz), dp(cs), dp(en), float(eng)))


def restart_branch(workdir, node=0):
    """The branch choice of CONTROL `restart` for node `node` (gcmc.f:353-394): a dict with the
    REVIVE to continue from (None: start from the CONFIG), the node's output directory and the
    number of branch entries found."""
    rev, out, prev = ctypes.create_string_buffer(4096), ctypes.create_string_buffer(4096), ctypes.c_int()
    rc = lib().fmc_restart_branch(str(workdir).encode(), int(node), rev, 4096, out, 4096, ctypes.byref(prev))
    check(rc if rc < 0 else 0)
    return {"revive": rev.value.decode() if rc == 1 else None, "outdir": out.value.decode(),
            "prevnodes": prev.value}


def _species_sites(deck_dir, g):
    """Sites per molecule of guest species g of a deck."""
    return _SITES_CACHE.setdefault((str(deck_dir), g), _read_sites(deck_dir, g))


_SITES_CACHE = {}


def _read_sites(deck_dir, g):
    # the FIELD guest blocks in order: the first ATOMS record after the g-th &guest header
    lines = open(os.path.join(str(deck_dir), "FIELD")).read().lower().splitlines()
    k = -1
    for i, line in enumerate(lines):
        if "&guest" in line:
            k += 1
            if k == g:
                for l2 in lines[i + 1:]:
                    if l2.strip().startswith("atoms"):
                        return int(l2.split()[1])
    raise ValueError("guest species not found in FIELD")


def read_revive(path, deck_dir):
    """A REVIVE as a dict: production, natms, chainstats, energy, guests (one (nmol, nsite, 3)
    array per species)."""
    info = deck_inspect(deck_dir)
    ng = info["nspecies"]
    nmol = np.zeros(max(ng, 1), dtype=np.int32)
    prod, natms = ctypes.c_int(0), ctypes.c_int(0)
    d, p = str(deck_dir).encode(), str(path).encode()
    check(lib().fmc_revive_read(p, d, None, ip(nmol), None, None, None, None))
    ns = [_read_sites(deck_dir, g) for g in range(ng)]
    xyz = np.zeros(max(1, sum(int(nmol[g]) * ns[g] * 3 for g in range(ng))))
    cs = np.zeros(1 + 14 * ng)
    en = np.zeros(max(ng, 1))
    check(lib().fmc_revive_read(p, d, ctypes.byref(prod), ip(nmol), dp(xyz), dp(cs), dp(en), ctypes.byref(natms)))
    guests, off = [], 0
    for g in range(ng):
        n = int(nmol[g]) * ns[g] * 3
        guests.append(xyz[off:off + n].reshape(int(nmol[g]), ns[g], 3))
        off += n
    return {"production": bool(prod.value), "natms": natms.value, "chainstats": cs, "energy": en[:ng],
            "guests": guests}
