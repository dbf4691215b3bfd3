"""ctypes binding of the FP64 CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs may import
this module.  The oracle is a restatement of FastMC 1.4.0's GCMC trial-move energy path
(ewald.f, vdw_terms.f, utility_pack.f, readinputs.f, gcmc.f) built from oracle/fmc_oracle.cpp
by oracle/Makefile; it is the checker, never the thing measured or shipped.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

MOVE_DTYPE = np.dtype([
    ("step", np.int32), ("iguest", np.int32), ("mtype", np.int32), ("randchoice", np.int32),
    ("accepted", np.int32), ("nmols_after", np.int32), ("pad0", np.int32), ("pad1", np.int32),
    ("ewld1", np.float64), ("ewld2", np.float64), ("ewld3", np.float64), ("vdw", np.float64),
    ("delrc", np.float64), ("estep", np.float64), ("rande", np.float64), ("energy_after", np.float64),
])

MV_INSERT, MV_DELETE, MV_DISPLACE = 1, 2, 3


def build():
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.orc_open.restype = vp
        L.orc_open.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ip]
        L.orc_close.argtypes = [vp]
        L.orc_last_error.restype = ctypes.c_char_p
        for name in ("orc_scalars",):
            getattr(L, name).argtypes = [vp, dp]
        L.orc_ints.argtypes = [vp, ip]
        L.orc_kvectors.argtypes = [vp, ip, dp]
        L.orc_sk.argtypes = [vp, dp, dp]
        L.orc_sknew.argtypes = [vp, dp, dp]
        L.orc_atoms.argtypes = [vp, dp, dp, ip, ip]
        L.orc_erc.argtypes = [vp, dp]
        L.orc_vvv.argtypes = [vp, ctypes.c_int, dp]
        L.orc_lstvdw.argtypes = [vp, ip]
        L.orc_guest_template.argtypes = [vp, ctypes.c_int, dp, dp, ip, dp]
        L.orc_ewald3en.restype = ctypes.c_double
        L.orc_ewald3en.argtypes = [vp, ctypes.c_int]
        L.orc_ewald1_guest.restype = ctypes.c_double
        L.orc_ewald1_guest.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, ctypes.c_int]
        L.orc_realspace.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp, ip, dp, dp, dp, dp]
        L.orc_run.restype = ctypes.c_int
        L.orc_run.argtypes = [vp, ctypes.c_int, ctypes.c_void_p]
        L.orc_run_to_completion.restype = ctypes.c_longlong
        L.orc_run_to_completion.argtypes = [vp, ctypes.c_longlong]
        L.orc_duni.restype = ctypes.c_double
        L.orc_duni.argtypes = [vp]
        L.orc_duni_stream.argtypes = [ctypes.c_int] * 5 + [dp]
        L.orc_guest_coords.argtypes = [vp, ctypes.c_int, dp]
        L.orc_load_guests.argtypes = [vp, ctypes.c_int, ctypes.c_int, dp]
        L.orc_stats.argtypes = [vp, ctypes.c_int, dp]
        L.orc_restart_flags.argtypes = [vp, ctypes.c_int, dp]
        L.orc_prob.argtypes = [vp, ctypes.c_int, ip, dp]
        L.orc_final_stats.argtypes = [vp, dp]
        L.orc_window_stats.argtypes = [vp, dp]
        L.orc_open_outputs.argtypes = [vp, ctypes.c_char_p]
        L.orc_pressures.argtypes = [vp, dp]
        assert L.orc_sizeof_moverec() == MOVE_DTYPE.itemsize
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"FastMC error {code}: {msg}")
        self.code = code


def duni_stream(seed, n):
    out = np.zeros(n)
    lib().orc_duni_stream(*[int(s) for s in seed], int(n), _dp(out))
    return out


class Chain:
    """One oracle chain opened from a CONTROL/FIELD/CONFIG directory."""

    def __init__(self, directory, seed=(12, 34, 56, 78)):
        L = lib()
        code = ctypes.c_int(0)
        self.h = L.orc_open(str(directory).encode(), *[int(s) for s in seed], ctypes.byref(code))
        if not self.h:
            raise OracleError(code.value, L.orc_last_error().decode())

    def close(self):
        if self.h:
            lib().orc_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # ---- introspection
    def scalars(self):
        out = np.zeros(15)
        lib().orc_scalars(self.h, _dp(out))
        keys = ["alpha", "rcut", "delr", "volm", "engunit", "temp", "beta", "drewd", "dlrpot", "spenergy",
                "dlpeng", "ewald1sum", "elrc", "energy", "statvolm"]
        return dict(zip(keys, out.tolist()))

    def ints(self):
        out = np.zeros(12, dtype=np.int32)
        lib().orc_ints(self.h, _ip(out))
        keys = ["imcon", "kmax1", "kmax2", "kmax3", "newld", "totatm", "ntpguest", "ntpatm", "mxgrid",
                "nframework", "gcmccount", "maxvdw"]
        return dict(zip(keys, [int(v) for v in out]))

    def kvectors(self):
        K = lib().orc_kvectors(self.h, None, None)
        lmn = np.zeros((K, 3), dtype=np.int32)
        akk = np.zeros(K)
        lib().orc_kvectors(self.h, _ip(lmn), _dp(akk))
        return lmn, akk

    def sk(self, new=False):
        K = self.ints()["newld"]
        re, im = np.zeros(K), np.zeros(K)
        (lib().orc_sknew if new else lib().orc_sk)(self.h, _dp(re), _dp(im))
        return re + 1j * im

    def atoms(self):
        n = self.ints()["totatm"]
        xyz, q = np.zeros((n, 3)), np.zeros(n)
        typ, frz = np.zeros(n, dtype=np.int32), np.zeros(n, dtype=np.int32)
        lib().orc_atoms(self.h, _dp(xyz), _dp(q), _ip(typ), _ip(frz))
        return xyz, q, typ, frz

    def erc(self):
        out = np.zeros(self.ints()["mxgrid"] + 1)
        lib().orc_erc(self.h, _dp(out))
        return out

    def vvv(self, k):
        out = np.zeros(self.ints()["mxgrid"] + 1)
        lib().orc_vvv(self.h, int(k), _dp(out))
        return out

    def lstvdw(self):
        nt = self.ints()["ntpatm"]
        out = np.zeros(nt * (nt + 1) // 2, dtype=np.int32)
        lib().orc_lstvdw(self.h, _ip(out))
        return out

    def guest_template(self, g=0):
        xyz, q, m = np.zeros((64, 3)), np.zeros(64), np.zeros(64)
        typ = np.zeros(64, dtype=np.int32)
        n = lib().orc_guest_template(self.h, int(g), _dp(xyz), _dp(q), _ip(typ), _dp(m))
        return xyz[:n].copy(), q[:n].copy(), typ[:n].copy(), m[:n].copy()

    def ewald3en(self, g=0):
        return lib().orc_ewald3en(self.h, int(g))

    def guest_coords(self, g=0):
        nmol = lib().orc_guest_coords(self.h, int(g), None)
        n = len(self.guest_template(g)[1])
        out = np.zeros((max(nmol * n, 1), 3))
        lib().orc_guest_coords(self.h, int(g), _dp(out))
        return out[: nmol * n].reshape(nmol, n, 3)

    # ---- energy routines
    def ewald1_guest(self, g, xyz, move, pass_=1):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        return lib().orc_ewald1_guest(self.h, int(g), xyz.shape[0], _dp(xyz), int(move), int(pass_))

    def realspace(self, g, xyz, ind=None, per_site=False):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        n = xyz.shape[0]
        ind = np.full(n, -1, dtype=np.int32) if ind is None else np.ascontiguousarray(ind, dtype=np.int32)
        e2, ev = ctypes.c_double(0), ctypes.c_double(0)
        se, sv = np.zeros(n), np.zeros(n)
        lib().orc_realspace(self.h, int(g), n, _dp(xyz), _ip(ind), ctypes.byref(e2), ctypes.byref(ev),
                            _dp(se), _dp(sv))
        if per_site:
            return se, sv
        return e2.value, ev.value

    def load_guests(self, g, xyz):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        nsite = len(self.guest_template(g)[1])
        return lib().orc_load_guests(self.h, int(g), xyz.shape[0] // nsite, _dp(xyz))

    # ---- move loop
    def run(self, n, trace=True):
        rec = np.zeros(n, dtype=MOVE_DTYPE) if trace else None
        r = lib().orc_run(self.h, int(n), rec.ctypes.data if trace else None)
        if r < 0:
            raise OracleError(-r, lib().orc_last_error().decode())
        return rec

    def run_to_completion(self, max_moves):
        return lib().orc_run_to_completion(self.h, int(max_moves))

    def duni(self):
        return lib().orc_duni(self.h)

    def final_stats(self):
        """The report's statistics (gcmc.f:1960-2037) as chainstats: [0] production moves, then
        per species 14 values (<N>,<E>,<EN>,<N^2>,<E^2>, 6th, errors of N,E,EN,N^2,E^2,Qst,Cv,6th)."""
        ng = self.ints()["ntpguest"]
        out = np.zeros(1 + 14 * ng)
        lib().orc_final_stats(self.h, _dp(out))
        return out

    def pressures(self):
        """Partial pressures (Pa) per guest and the pressure-equilibration tolerance still in
        force (0 once the pressures have equilibrated)."""
        ng = self.ints()["ntpguest"]
        out = np.zeros(ng + 1)
        lib().orc_pressures(self.h, _dp(out))
        return out[:ng], float(out[ng])

    def open_outputs(self, directory):
        """numguests.out (every nnumg moves) and his.xyz (CONTROL `history`) into `directory`;
        None closes them."""
        r = lib().orc_open_outputs(self.h, None if directory is None else str(directory).encode())
        if r:
            raise OracleError(-r, "cannot open the output files")

    def window_stats(self):
        """Averaging-window state (gcmc.f:1814-1928): avcount, rollcount, window sums, variances,
        current means (8 per species) and selectivities."""
        ng = self.ints()["ntpguest"]
        out = np.zeros(2 + 24 * ng + ng * ng)
        lib().orc_window_stats(self.h, _dp(out))
        o = out[2:]
        return {"avcount": int(out[0]), "rollcount": int(out[1]), "sum": o[:8 * ng].reshape(ng, 8),
                "var": o[8 * ng:16 * ng].reshape(ng, 8), "avg": o[16 * ng:24 * ng].reshape(ng, 8),
                "seltot": o[24 * ng:24 * ng + ng * ng].reshape(ng, ng)}

    def prob(self):
        """Probability grids (storeprob): array [plots, na, nb, nc] of binned weights."""
        dims = np.zeros(4, dtype=np.int32)
        lib().orc_prob(self.h, 0, _ip(dims), None)
        n, na, nb, nc = (int(v) for v in dims)
        out = np.zeros((n, na, nb, nc))
        for k in range(n):
            buf = np.zeros(na * nb * nc)
            lib().orc_prob(self.h, k, None, _dp(buf))
            out[k] = buf.reshape(na, nb, nc)
        return out

    def restart_flags(self, production, chainstats):
        """Production flag and chain statistics of a restart from REVIVE (after load_guests)."""
        cs = np.ascontiguousarray(chainstats, dtype=np.float64)
        lib().orc_restart_flags(self.h, int(production), _dp(cs))

    def stats(self, g=0):
        out = np.zeros(6)
        lib().orc_stats(self.h, int(g), _dp(out))
        return dict(zip(["N", "E", "EN", "N2", "E2", "prodcount"], out.tolist()))
