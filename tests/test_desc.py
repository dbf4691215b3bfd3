"""Systems handed over as arrays (fmc_system_desc) on the host: a deck read into a descriptor
builds bit-identical tables to the deck itself; a descriptor built from the generator's own
arrays builds the same k-vectors and tables; malformed descriptors fail with the reference's
error codes before any device work."""
import ctypes

import numpy as np
import pytest

from desc_util import desc_from_synth


def _inspect_desc(fmc, d):
    from fastmc_b200 import _lib

    L = _lib.lib()
    K, nerc, nt = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    ints, dbls = np.zeros(16, dtype=np.int32), np.zeros(16)
    _lib.check(L.fmc_desc_inspect(ctypes.byref(d.s), _lib.ip(ints), _lib.dp(dbls), None, None, None, None,
                                  ctypes.byref(K), ctypes.byref(nerc), None, ctypes.byref(nt)))
    lmn, akk = np.zeros((K.value, 3), dtype=np.int32), np.zeros(K.value)
    erc, q = np.zeros(nerc.value), np.zeros(max(int(ints[9]), 1))
    vvv = np.zeros(nt.value * nerc.value)
    _lib.check(L.fmc_desc_inspect(ctypes.byref(d.s), None, None, _lib.ip(lmn), _lib.dp(akk), _lib.dp(erc),
                                  _lib.dp(q), ctypes.byref(K), ctypes.byref(nerc), _lib.dp(vvv), ctypes.byref(nt)))
    return ints, dbls, lmn, akk, erc, q[: int(ints[9])], vvv.reshape(nt.value, nerc.value)


def test_descriptor_struct_layout_matches_the_library(fmc):
    from fastmc_b200 import _lib

    sz = np.zeros(3, dtype=np.int32)
    _lib.check(_lib.lib().fmc_desc_sizes(_lib.ip(sz)))
    assert list(sz) == [ctypes.sizeof(_lib.SystemDescStruct), ctypes.sizeof(_lib.GuestDesc),
                        ctypes.sizeof(_lib.VdwDesc)]


@pytest.mark.parametrize("deck", ["small", "mixture", "forms", "calf20", "imcon4", "binary_preloaded"])
def test_deck_read_into_a_descriptor_builds_identical_tables(fmc, decks, deck):
    d = decks[deck]
    info = fmc.deck_inspect(d)
    desc = fmc.SystemDesc.from_deck(d)
    ints, dbls, lmn, akk, erc, q, vvv = _inspect_desc(fmc, desc)
    ref_ints = [info[k] for k in ("imcon", "kmax1", "kmax2", "kmax3", "K", "natoms", "nspecies", "ntypes", "mxgrid",
                                  "nframework")]
    assert list(ints[:10]) == ref_ints
    for k, v in zip(("alpha", "rcut", "delr", "volm", "engunit", "temp", "beta", "drewd", "dlrpot"), dbls[:9]):
        assert v == info[k], k
    assert np.array_equal(lmn, info["lmn"]) and np.array_equal(akk, info["akk"])
    assert np.array_equal(erc, info["erc"]) and np.array_equal(q, info["charges"])
    tabs = fmc.deck_vdw(d)
    assert len(tabs) == vvv.shape[0]
    for a, b in zip(tabs, vvv):
        assert np.array_equal(a, b)
    desc.free()


def test_descriptor_from_generator_arrays_matches_its_deck(fmc, decks):
    from fastmc_b200 import synth

    fw = synth.plain_small_framework()
    desc = desc_from_synth(fmc, fw, synth.CO2, 0.15, 298.0, (8, 8, 8))
    ints, dbls, lmn, akk, erc, q, vvv = _inspect_desc(fmc, desc)
    info = fmc.deck_inspect(decks["small"])
    assert ints[4] == info["K"] and np.array_equal(lmn, info["lmn"])
    assert np.allclose(akk, info["akk"], rtol=1e-12, atol=0) and np.allclose(erc, info["erc"], rtol=1e-12, atol=0)
    assert np.allclose(q, info["charges"], rtol=0, atol=1e-10)  # the deck prints 10 decimals
    tabs = fmc.deck_vdw(decks["small"])
    for a, b in zip(tabs, vvv):
        assert np.allclose(a, b, rtol=1e-12, atol=1e-12 * np.max(np.abs(a)))


def test_malformed_descriptors_fail_with_the_reference_codes(fmc):
    from fastmc_b200 import _lib, synth

    fw = synth.plain_small_framework()
    h = ctypes.c_void_p()
    seed = np.array([1, 2, 3, 4], dtype=np.int32)

    def code(desc):
        rc = _lib.lib().fmc_chain_create(ctypes.byref(desc.s), _lib.ip(seed), 0, ctypes.byref(h))
        return rc, _lib.lib().fmc_last_error().decode()

    big = desc_from_synth(fmc, fw, synth.CO2, 0.15, 298.0, (8, 8, 8), rcut=13.5)  # a/2 = 12.916
    assert code(big)[0] == 95
    bad_cell = desc_from_synth(fmc, fw, synth.CO2, 0.15, 298.0, (8, 8, 8))
    bad_cell.s.cell[4] = 26.5  # imcon 1 needs a cube
    assert code(bad_cell)[0] == 410
    bad_type = desc_from_synth(fmc, fw, synth.CO2, 0.15, 298.0, (8, 8, 8))
    bad_type.s.vdw[0].type_i = 99
    assert code(bad_type)[0] == 4
    no_pbc = desc_from_synth(fmc, fw, synth.CO2, 0.15, 298.0, (8, 8, 8))
    no_pbc.s.imcon = 0
    assert code(no_pbc)[0] == -4
    cold = desc_from_synth(fmc, fw, synth.CO2, 0.15, 0.0, (8, 8, 8))
    assert code(cold)[0] == 380
