"""The no-allocation reciprocal pass against the chain's own reciprocal pass.

fmc_ewald1_guest_noalloc serves callers that may not allocate GPU memory themselves; the
buffers it works on belong to the caller (here: torch tensors standing in for the caller's
pool).  Two calls in a row (an insertion, then a fused displacement) must give the same pass
energy and S_new as fmc_ewald1_guest on the same state, within the FP64 tolerance used by the
other parity tests (1e-9 relative); so must a deletion issued on the caller's own stream, and a
pass whose phase tables need more than 48 KB of shared memory (against a direct FP64 sum).  This file sorts last so a stop-at-first-failure run has
already run every other test.
"""
import ctypes
import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
REL = 1e-9
R4PIE0 = 138935.4835


def _cell(deck):
    lines = open(os.path.join(deck, "CONFIG")).read().split("\n")
    return np.array([[float(v) for v in lines[k].split()] for k in (2, 3, 4)])


def test_noalloc_pass_matches_chain_pass_twice(fmc, oracle_mod, decks):
    import torch

    from fastmc_b200 import _lib

    deck = decks["small"]
    chain = fmc.Chain(deck, seed=(3, 5, 7, 11))
    chain.run(400, trace=False)  # some guests present, so S(k) is not the framework's alone
    info = chain.info()
    lmn, akk = chain.kvectors()
    sk = chain.sk()
    K = len(akk)
    dev = torch.device("cuda", 0)
    d_lmn = torch.tensor(lmn.reshape(-1), dtype=torch.int32, device=dev)
    d_akk = torch.tensor(akk, dtype=torch.float64, device=dev)
    d_sk = torch.tensor(np.stack([sk.real, sk.imag], axis=1).reshape(-1), dtype=torch.float64, device=dev)
    d_new = torch.zeros(2 * K, dtype=torch.float64, device=dev)
    d_e = torch.zeros(1, dtype=torch.float64, device=dev)
    kmax = np.array([info["kmax1"], info["kmax2"], info["kmax3"]], dtype=np.int32)
    cell = np.ascontiguousarray(_cell(deck).reshape(-1))
    tmpl, q, _, _ = oracle_mod.Chain(deck).guest_template(0)
    recip_pref = 2.0 * (2.0 * math.pi / info["volm"]) * R4PIE0
    engsic = -R4PIE0 * info["alpha"] * float(np.sum(q * q)) / 1.7724538509055159
    L = _lib.lib()
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731

    def call(move, old, new):
        sites = np.concatenate([np.c_[old, q] if old is not None else np.zeros((0, 4)),
                                np.c_[new, q] if new is not None else np.zeros((0, 4))]).reshape(-1)
        sites = np.ascontiguousarray(sites, dtype=np.float64)
        nold = 0 if old is None else len(old)
        nnew = 0 if new is None else len(new)
        rc = L.fmc_ewald1_guest_noalloc(K, _lib.ip(kmax), _lib.dp(cell), ptr(d_lmn), ptr(d_akk), ptr(d_sk), move,
                                        nold, nnew, _lib.dp(sites), recip_pref, engsic, ptr(d_new), ptr(d_e), None)
        assert rc == 0, L.fmc_last_error().decode()
        torch.cuda.synchronize()
        snew = d_new.cpu().numpy().reshape(-1, 2)
        return float(d_e.cpu().item()), snew[:, 0] + 1j * snew[:, 1]

    # call 1: an insertion
    rng = np.random.default_rng(9)
    new = tmpl + rng.uniform(0, 1, 3) @ _cell(deck)
    e_na, s_na = call(fmc.INSERT, None, new)
    e_ch = chain.ewald1_guest(0, new, fmc.INSERT)
    s_ch = chain.sk(pending=True)
    assert abs(e_na - e_ch) <= REL * abs(e_ch)
    assert np.max(np.abs(s_na - s_ch)) <= REL * np.max(np.abs(s_ch))
    # call 2, straight after: a fused displacement of an existing molecule
    old = chain.guest_coords(0)[0]
    new2 = old + np.array([0.3, -0.2, 0.1])
    e_na2, s_na2 = call(fmc.DISPLACE, old, new2)
    chain.ewald1_guest(0, old, fmc.DISPLACE, 1)
    e_ch2 = chain.ewald1_guest(0, new2, fmc.DISPLACE, 2)
    s_ch2 = chain.sk(pending=True)
    assert abs(e_na2 - e_ch2) <= REL * max(abs(e_ch2), 1e-6)
    assert np.max(np.abs(s_na2 - s_ch2)) <= REL * np.max(np.abs(s_ch2))


def _noalloc(L, lib, K, kmax, cell, d_lmn, d_akk, d_sk, move, sites, nold, nnew, recip_pref, engsic, d_new, d_e,
             stream=None):
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    s = np.ascontiguousarray(np.asarray(sites, dtype=np.float64).reshape(-1))
    k = np.ascontiguousarray(np.asarray(kmax, dtype=np.int32))
    c = np.ascontiguousarray(np.asarray(cell, dtype=np.float64).reshape(-1))
    rc = L.fmc_ewald1_guest_noalloc(K, lib.ip(k), lib.dp(c), ptr(d_lmn), ptr(d_akk), ptr(d_sk), move, nold, nnew,
                                    lib.dp(s), recip_pref, engsic, ptr(d_new), ptr(d_e), stream)
    assert rc == 0, L.fmc_last_error().decode()


def test_noalloc_delete_on_a_stream_and_a_wide_phase_table(fmc, oracle_mod, decks):
    """A deletion on a caller's own stream against the chain's pass; then, on the 3392-atom deck
    (kmax 12), 80 sites whose phase tables need more than 48 KB of shared memory against a
    direct FP64 sum; then a kmax smaller than the k-vector table's, which must give NaN."""
    import torch

    from fastmc_b200 import _lib

    L = _lib.lib()
    dev = torch.device("cuda", 0)
    deck = decks["small"]
    chain = fmc.Chain(deck, seed=(2, 3, 5, 7))
    chain.run(400, trace=False)
    info = chain.info()
    lmn, akk = chain.kvectors()
    sk = chain.sk()
    K = len(akk)
    d_lmn = torch.tensor(lmn.reshape(-1), dtype=torch.int32, device=dev)
    d_akk = torch.tensor(akk, dtype=torch.float64, device=dev)
    d_sk = torch.tensor(np.stack([sk.real, sk.imag], axis=1).reshape(-1), dtype=torch.float64, device=dev)
    d_new = torch.zeros(2 * K, dtype=torch.float64, device=dev)
    d_e = torch.zeros(1, dtype=torch.float64, device=dev)
    tmpl, q, _, _ = oracle_mod.Chain(deck).guest_template(0)
    recip_pref = 2.0 * (2.0 * math.pi / info["volm"]) * R4PIE0
    engsic = -R4PIE0 * info["alpha"] * float(np.sum(q * q)) / 1.7724538509055159
    old = chain.guest_coords(0)[0]
    stream = torch.cuda.Stream(device=dev)
    _noalloc(L, _lib, K, [info["kmax1"], info["kmax2"], info["kmax3"]], _cell(deck), d_lmn, d_akk, d_sk, fmc.DELETE,
             np.c_[old, q], len(old), 0, recip_pref, engsic, d_new, d_e, ctypes.c_void_p(stream.cuda_stream))
    stream.synchronize()
    e_na = float(d_e.cpu().item())
    s_na = d_new.cpu().numpy().reshape(-1, 2)
    e_ch = chain.ewald1_guest(0, old, fmc.DELETE)
    s_ch = chain.sk(pending=True)
    assert abs(e_na - e_ch) <= REL * abs(e_ch)
    assert np.max(np.abs((s_na[:, 0] + 1j * s_na[:, 1]) - s_ch)) <= REL * np.max(np.abs(s_ch))
    chain.close()

    # 40 old + 40 new sites on the kmax-12 deck: 80 x 39 x 16 B = 49,920 B of phase tables
    big = decks["large"]
    c2 = fmc.Chain(big, seed=(1, 1, 2, 3))
    inf2 = c2.info()
    lmn2, akk2 = c2.kvectors()
    sk2 = c2.sk()
    K2 = len(akk2)
    cell2 = _cell(big)
    rng = np.random.default_rng(17)
    pos = rng.uniform(0, 1, (80, 3)) @ cell2
    qs = np.where(np.arange(80) % 3 == 0, 0.7, -0.35)
    d_lmn2 = torch.tensor(lmn2.reshape(-1), dtype=torch.int32, device=dev)
    d_akk2 = torch.tensor(akk2, dtype=torch.float64, device=dev)
    d_sk2 = torch.tensor(np.stack([sk2.real, sk2.imag], axis=1).reshape(-1), dtype=torch.float64, device=dev)
    d_new2 = torch.zeros(2 * K2, dtype=torch.float64, device=dev)
    pref2 = 2.0 * (2.0 * math.pi / inf2["volm"]) * R4PIE0
    kmax2 = [inf2["kmax1"], inf2["kmax2"], inf2["kmax3"]]
    assert 80 * (sum(kmax2) + 3) * 16 > 48 * 1024
    _noalloc(L, _lib, K2, kmax2, cell2, d_lmn2, d_akk2, d_sk2, fmc.DISPLACE, np.c_[pos, qs], 40, 40, pref2, 0.0,
             d_new2, d_e)
    torch.cuda.synchronize()
    e_big = float(d_e.cpu().item())
    s_big = d_new2.cpu().numpy().reshape(-1, 2)
    # direct FP64 sum: S_new = S - sum_old q e^{i 2 pi lmn.s} + sum_new q e^{i 2 pi lmn.s}
    frac = pos @ np.linalg.inv(cell2)
    terms = qs[:, None] * np.exp(2j * np.pi * (frac @ lmn2.T))
    sn_ref = sk2 - terms[:40].sum(0) + terms[40:].sum(0)
    e_ref = pref2 * float(np.sum(akk2 * (np.abs(sn_ref) ** 2 - np.abs(sk2) ** 2)))
    scale = pref2 * float(np.sum(akk2 * (np.abs(sn_ref) ** 2 + np.abs(sk2) ** 2)))
    assert abs(e_big - e_ref) <= REL * max(abs(e_ref), 1e-3 * scale)
    assert np.max(np.abs((s_big[:, 0] + 1j * s_big[:, 1]) - sn_ref)) <= REL * np.max(np.abs(sn_ref))

    # a declared kmax below the table's: the out-of-range k-vectors make the energy NaN
    _noalloc(L, _lib, K2, [8, 8, 8], cell2, d_lmn2, d_akk2, d_sk2, fmc.DISPLACE, np.c_[pos[:2], qs[:2]], 1, 1, pref2,
             0.0, d_new2, d_e)
    torch.cuda.synchronize()
    assert math.isnan(float(d_e.cpu().item()))
    c2.close()


def test_noalloc_rejects_sizes_beyond_its_scratch(fmc):
    from fastmc_b200 import _lib

    L = _lib.lib()
    kmax = np.array([8, 8, 8], dtype=np.int32)
    cell = np.eye(3).reshape(-1) * 25.0
    sites = np.zeros(4)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = L.fmc_ewald1_guest_noalloc(40000, _lib.ip(kmax), _lib.dp(cell), dummy, dummy, dummy, fmc.INSERT, 0, 1,
                                    _lib.dp(sites), 1.0, 0.0, dummy, dummy, None)
    assert rc == -7
    assert "maximum" in L.fmc_last_error().decode()
