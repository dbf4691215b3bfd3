"""ctypes binding of libfastmc_b200.so (the C ABI declared in include/fastmc_b200.h).

The library is built in-tree by fastmc-1.4.0_b200/build.py.  There is no fallback: if the
shared library is missing or fails to load, every call raises.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG, "lib", "libfastmc_b200.so")

MOVE_DTYPE = np.dtype([
    ("step", np.int32), ("iguest", np.int32), ("mtype", np.int32), ("randchoice", np.int32),
    ("accepted", np.int32), ("nmols_after", np.int32), ("pad0", np.int32), ("pad1", np.int32),
    ("ewld1", np.float64), ("ewld2", np.float64), ("ewld3", np.float64), ("vdw", np.float64),
    ("delrc", np.float64), ("estep", np.float64), ("rande", np.float64), ("energy_after", np.float64),
])

INSERT, DELETE, DISPLACE, TRANSLATE, ROTATE, JUMP, NOOP, MULTIJUMP = 1, 2, 3, 4, 5, 6, 7, 8  # NOOP: flex / swap

class GuestDesc(ctypes.Structure):
    """fmc_guest_desc of the C ABI."""
    _fields_ = [("name", ctypes.c_char_p), ("nsite", ctypes.c_int), ("site_name", ctypes.POINTER(ctypes.c_char_p)),
                ("mass", ctypes.POINTER(ctypes.c_double)), ("charge", ctypes.POINTER(ctypes.c_double)),
                ("tx", ctypes.POINTER(ctypes.c_double)), ("ty", ctypes.POINTER(ctypes.c_double)),
                ("tz", ctypes.POINTER(ctypes.c_double)), ("type", ctypes.POINTER(ctypes.c_int)),
                ("nmols", ctypes.c_int), ("xyz", ctypes.POINTER(ctypes.c_double)), ("pressure_pa", ctypes.c_double),
                ("move_freq", ctypes.c_double * 9), ("disp_ratio", ctypes.c_double), ("tran_ratio", ctypes.c_double)]


class VdwDesc(ctypes.Structure):
    """fmc_vdw_desc of the C ABI."""
    _fields_ = [("type_i", ctypes.c_int), ("type_j", ctypes.c_int), ("form", ctypes.c_int),
                ("prm", ctypes.c_double * 5)]


class SystemDescStruct(ctypes.Structure):
    """fmc_system_desc of the C ABI."""
    _fields_ = [("imcon", ctypes.c_int), ("cell", ctypes.c_double * 9), ("alpha", ctypes.c_double),
                ("kmax", ctypes.c_int * 3), ("rcut", ctypes.c_double), ("rvdw", ctypes.c_double),
                ("delr", ctypes.c_double), ("engunit", ctypes.c_double), ("ntypes", ctypes.c_int),
                ("type_names", ctypes.POINTER(ctypes.c_char_p)), ("nframework", ctypes.c_int),
                ("fw_xyz", ctypes.POINTER(ctypes.c_double)), ("fw_charge", ctypes.POINTER(ctypes.c_double)),
                ("fw_type", ctypes.POINTER(ctypes.c_int)), ("fw_mass", ctypes.POINTER(ctypes.c_double)),
                ("nguest", ctypes.c_int), ("guests", ctypes.POINTER(GuestDesc)), ("nvdw", ctypes.c_int),
                ("vdw", ctypes.POINTER(VdwDesc)), ("temperature", ctypes.c_double), ("eq_steps", ctypes.c_int),
                ("prod_steps", ctypes.c_int), ("max_guest_atoms", ctypes.c_int),
                ("averaging_window", ctypes.c_int), ("acceptance_sampling", ctypes.c_int),
                ("rota_ratio", ctypes.c_double), ("owner", ctypes.c_void_p)]


# Every function the C ABI exports: name -> (restype, argtypes)
_vp, _ip, _dp, _ci, _cd = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), \
    ctypes.c_int, ctypes.c_double
SIGNATURES = {
    "fmc_version": (_ci, []),
    "fmc_last_error": (ctypes.c_char_p, []),
    "fmc_chain_open": (_ci, [ctypes.c_char_p, _ip, _ci, ctypes.POINTER(_vp)]),
    "fmc_chain_open_node": (_ci, [ctypes.c_char_p, _ip, _ci, _ci, ctypes.POINTER(_vp)]),
    "fmc_restart_branch": (_ci, [ctypes.c_char_p, _ci, ctypes.c_char_p, _ci, ctypes.c_char_p, _ci, _ip]),
    "fmc_chain_resident": (_ci, [_vp, _ci, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
    "fmc_chain_close": (None, [_vp]),
    "fmc_chain_create": (_ci, [ctypes.POINTER(SystemDescStruct), _ip, _ci, ctypes.POINTER(_vp)]),
    "fmc_deck_describe": (_ci, [ctypes.c_char_p, ctypes.POINTER(SystemDescStruct)]),
    "fmc_desc_free": (None, [ctypes.POINTER(SystemDescStruct)]),
    "fmc_desc_sizes": (_ci, [_ip]),
    "fmc_desc_inspect": (_ci, [ctypes.POINTER(SystemDescStruct), _ip, _dp, _ip, _dp, _dp, _dp, _ip, _ip, _dp, _ip]),
    "fmc_ewald1_guest_xyz": (_ci, [_vp, _ci, _ci, _dp, _dp, _dp, _ci, _ci, _dp]),
    "fmc_guest_realspace_xyz": (_ci, [_vp, _ci, _ci, _dp, _dp, _dp, _ci, _dp, _dp]),
    "fmc_commit_xyz": (_ci, [_vp, _ci, _ci, _ci, _dp, _dp, _dp]),
    "fmc_chain_info": (_ci, [_vp, _ip, _dp]),
    "fmc_ewald1": (_ci, [_vp, _dp, _ip]),
    "fmc_ewald1_guest": (_ci, [_vp, _ci, _ci, _dp, _ci, _ci, _dp]),
    "fmc_guest_realspace": (_ci, [_vp, _ci, _ci, _dp, _ci, _dp, _dp]),
    "fmc_commit": (_ci, [_vp, _ci, _ci, _ci, _dp]),
    "fmc_reject": (_ci, [_vp]),
    "fmc_set_guests": (_ci, [_vp, _ci, _ci, _dp]),
    "fmc_single_point": (_ci, [_vp, _dp, _dp]),
    "fmc_get_sk": (_ci, [_vp, _ci, _dp, _dp]),
    "fmc_kvectors": (_ci, [_vp, _ip, _dp]),
    "fmc_run": (_ci, [_vp, _ci, _vp]),
    "fmc_guest_coords": (_ci, [_vp, _ci, _dp, _ip, _ip]),
    "fmc_stats": (_ci, [_vp, _ci, _dp]),
    "fmc_chain_profile": (_ci, [_vp, _ci, _dp]),
    "fmc_run_timed": (_ci, [_vp, _ci, _vp, ctypes.POINTER(ctypes.c_float)]),
    "fmc_ewald1_guest_noalloc": (_ci, [_ci, _ip, _dp, _vp, _vp, _vp, _ci, _ci, _ci, _dp, _cd, _cd, _vp, _vp, _vp]),
    "fmc_batch_open": (_ci, [_ci, ctypes.POINTER(ctypes.c_char_p), _ip, _ci, ctypes.POINTER(_vp)]),
    "fmc_batch_open_edge": (_ci, [_ci, ctypes.POINTER(ctypes.c_char_p), _ip, _ci, ctypes.c_double,
                                  ctypes.POINTER(_vp)]),
    "fmc_batch_autotune": (_ci, [_ci, ctypes.POINTER(ctypes.c_char_p), _ip, _ci, _dp, _ci, _ci, _dp,
                                 ctypes.POINTER(ctypes.c_float)]),
    "fmc_batch_autotune_tiles": (_ci, [_ci, ctypes.POINTER(ctypes.c_char_p), _ip, _ci, ctypes.c_double, _ip, _ci, _ci,
                                       _ci, _ip, ctypes.POINTER(ctypes.c_float)]),
    "fmc_batch_tiles": (_ci, [_ip, _ip, _ip, _ci]),
    "fmc_batch_set_tile": (_ci, [_vp, _ci]),
    "fmc_batch_get_tile": (_ci, [_vp]),
    "fmc_batch_close": (None, [_vp]),
    "fmc_batch_run": (_ci, [_vp, _ci, _vp, ctypes.POINTER(ctypes.c_float)]),
    "fmc_batch_profile": (_ci, [_vp, _ci]),
    "fmc_batch_chain_state": (_ci, [_vp, _ci, _dp]),
    "fmc_batch_chain_timing": (_ci, [_vp, _ci, ctypes.POINTER(ctypes.c_longlong)]),
    "fmc_batch_voxels": (_ci, [_vp, _ci, _ip, _ip, _ip, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)]),
    "fmc_batch_guest_coords": (_ci, [_vp, _ci, _ci, _dp, _ip, _ip]),
    "fmc_revive_write_state": (_ci, [ctypes.c_char_p, ctypes.c_char_p, _ci, _ip, _dp, _dp, _dp, ctypes.c_double]),
    "fmc_revive_read": (_ci, [ctypes.c_char_p, ctypes.c_char_p, _ip, _ip, _dp, _dp, _dp, _ip]),
    "fmc_chain_write_revive": (_ci, [_vp, ctypes.c_char_p]),
    "fmc_chain_restart": (_ci, [_vp, ctypes.c_char_p]),
    "fmc_batch_write_revive": (_ci, [_vp, _ci, ctypes.c_char_p]),
    "fmc_batch_restart": (_ci, [_vp, _ci, ctypes.c_char_p]),
    "fmc_chain_prob": (_ci, [_vp, _ci, _ip, _dp]),
    "fmc_chain_open_outputs": (_ci, [_vp, ctypes.c_char_p]),
    "fmc_chain_pressures": (_ci, [_vp, _dp]),
    "fmc_batch_pressures": (_ci, [_vp, _ci, _dp]),
    "fmc_batch_write_numguests": (_ci, [_vp, _ci, _vp, _ci, ctypes.c_char_p, _ci]),
    "fmc_chain_window_stats": (_ci, [_vp, _dp]),
    "fmc_chain_final_stats": (_ci, [_vp, _dp]),
    "fmc_chain_write_report": (_ci, [_vp, ctypes.c_char_p]),
    "fmc_write_report": (_ci, [ctypes.c_char_p, _dp, _dp, ctypes.c_char_p]),
    "fmc_batch_window_stats": (_ci, [_vp, _ci, _dp]),
    "fmc_batch_control_block_bytes": (_ci, []),
    "fmc_system_block_bytes": (_ci, []),
    "fmc_batch_final_stats": (_ci, [_vp, _ci, _dp]),
    "fmc_batch_write_report": (_ci, [_vp, _ci, ctypes.c_char_p]),
    "fmc_write_prob_cube": (_ci, [ctypes.c_char_p, ctypes.c_char_p, _dp, ctypes.c_longlong]),
    "fmc_atomic_number": (_ci, [ctypes.c_double]),
    "fmc_chain_write_prob": (_ci, [_vp, ctypes.c_char_p]),
    "fmc_batch_prob": (_ci, [_vp, _ci, _ci, _ip, _dp]),
    "fmc_batch_write_prob": (_ci, [_vp, _ci, ctypes.c_char_p]),
    "fmc_server_open": (_ci, [_ci, _ci, ctypes.c_longlong, _ci, ctypes.POINTER(_vp)]),
    "fmc_server_close": (None, [_vp]),
    "fmc_server_submit": (_ci, [_vp, ctypes.c_char_p, _ip, ctypes.c_longlong, _ip]),
    "fmc_server_cancel": (_ci, [_vp, _ci]),
    "fmc_server_keep_final_state": (_ci, [_vp, _ci]),
    "fmc_server_write_revive": (_ci, [_vp, _ci, ctypes.c_char_p]),
    "fmc_server_step": (_ci, [_vp, _ci, _ip, _ip, ctypes.POINTER(ctypes.c_float)]),
    "fmc_server_poll": (_ci, [_vp, _ci, _ip, _dp]),
    "fmc_server_busy": (_ci, [_vp, _ip]),
    "fmc_server_poll_done": (_ci, [_vp, _ip, _ip, _dp, _ci, _ip]),
    "fmc_server_stats": (_ci, [_vp, _dp]),
    "fmc_server_set_voxel_edge": (_ci, [_vp, ctypes.c_double]),
    "fmc_deck_footprint": (_ci, [ctypes.c_char_p, ctypes.c_double, ctypes.POINTER(ctypes.c_longlong),
                                 ctypes.POINTER(ctypes.c_double)]),
    "fmc_server_memory": (_ci, [_vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
    "fmc_deck_vdw": (_ci, [ctypes.c_char_p, _ci, _dp, _ip]),
    "fmc_deck_inspect": (_ci, [ctypes.c_char_p, _ip, _dp, _ip, _dp, _dp, _dp, _ip, _ip]),
    "fmc_deck_voxels": (_ci, [ctypes.c_char_p, ctypes.c_double, _ip, _ip, _ip, ctypes.c_longlong,
                              ctypes.POINTER(ctypes.c_longlong)]),
}

_lib = None


class FastMCError(RuntimeError):
    """Error returned by the library; `code` is the reference's error code when > 0."""

    def __init__(self, code, msg):
        super().__init__(f"FastMC error {code}: {msg}")
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FastMCError(-1, f"{LIB_PATH} is missing; build it with fastmc-1.4.0_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        raise FastMCError(rc, lib().fmc_last_error().decode())
    return rc


def dp(a):
    return a.ctypes.data_as(_dp)


def ip(a):
    return a.ctypes.data_as(_ip)
