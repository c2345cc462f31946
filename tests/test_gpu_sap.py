"""SAP digit decomposition on the GPU (tp_sap_decompose_batch): bit-exact against the
reference's recorded outputs (tests/golden/sap.*), in batches that mix digit counts and
accumulator resets, and decrypting like the reference's tests/sap_decomposer_tests.cpp
TestDecomp (digit i rounds to the message's i-th radix digit)."""
from __future__ import annotations

import ctypes
import json
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import CGGI_BINARY, P, lwe_secret, rlwe_secret, sha256, sm64

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLD))
from make_sap_golden import case_inputs  # noqa: E402

MANIFEST = json.loads((GOLD / "sap.json").read_text())


def decomposer(c, keys, beta, restart):
    from fhetoothpaste_b200 import GpuSAPDecomposer
    return GpuSAPDecomposer((c["variant"], c["N"], c["n"], 1 << c["rotation"][0], c["rotation"][1]),
                            (1 << c["trace"][0], c["trace"][1]), (1 << c["ks"][0], c["ks"][1]), *keys,
                            hamming_weight=beta, restart_period=restart)


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_matches_reference_outputs(native, oracle, cuda, name):
    c = MANIFEST[name]
    N, n = c["N"], c["n"]
    sk = lwe_secret(c["variant"], n, N, seed=c["sk_seed"])
    z = rlwe_secret(N, seed=c["sk_seed"] + 1)
    keys = oracle.sap_keygen(c["variant"], N, n, tuple(c["rotation"]), tuple(c["trace"]), tuple(c["ks"]), c["std"],
                             sk, z, c["key_seed"])
    assert [sha256(k) for k in keys] == c["key_sha256"]
    dec = decomposer(c, keys, c["beta"], c["restart"])
    lwes = case_inputs(n, c["bits"], c["count"], c["in_seed"])
    digits, got = dec.Decompose(lwes, c["radix"], c["out_digits"])
    assert [sha256(g) for g in got] == c["output_sha256"]
    whole = np.load(GOLD / "sap.npz")
    if name in whole.files:
        np.testing.assert_array_equal(got, whole[name])
    for j in range(c["count"]):   # the digit count is where the reference's output stops
        nz = [d for d in range(c["out_digits"]) if got[j, d].any()]
        assert not nz or max(nz) < digits[j]


@pytest.mark.parametrize("name", sorted(k for k, c in MANIFEST.items() if c["N"] <= 1024))
def test_homtrunc_and_reset_match_reference(native, oracle, cuda, name):
    """HomTrunc and ResetAccumulator as their own calls, on the recorded random inputs; then a batch
    of both against the oracle, with ResetAccumulator at a nonzero radix too."""
    from oracle.oracle import random_acc
    c = MANIFEST[name]
    N, n = c["N"], c["n"]
    sk = lwe_secret(c["variant"], n, N, seed=c["sk_seed"])
    z = rlwe_secret(N, seed=c["sk_seed"] + 1)
    keys = oracle.sap_keygen(c["variant"], N, n, tuple(c["rotation"]), tuple(c["trace"]), tuple(c["ks"]), c["std"],
                             sk, z, c["key_seed"])
    dec = decomposer(c, keys, c["beta"], c["restart"])
    x = random_acc(N, 2, c["in_seed"] + 1)
    assert sha256(dec.HomTrunc(x[0], c["radix"])[0]) == c["homtrunc_sha256"]
    assert sha256(dec.ResetAccumulator(x[1], 0)[0]) == c["reset_sha256"]
    y = random_acc(N, 5, c["in_seed"] + 7)
    ht = dec.HomTrunc(y, c["radix"])
    rs = dec.ResetAccumulator(y, c["radix"])
    for j in (0, 4):
        np.testing.assert_array_equal(ht[j], oracle.sap_homtrunc(N, tuple(c["trace"]), keys[1], c["radix"], y[j]))
        np.testing.assert_array_equal(rs[j], oracle.sap_reset(c["variant"], N, n, tuple(c["rotation"]), keys[0],
                                                              tuple(c["ks"]), keys[2], c["radix"], y[j]))


def test_radix_extremes_against_oracle(native, oracle, cuda):
    """Radix 2 (the deepest tree; the reference's own buffer is too small for it) and radix N
    (no tree: the whole trace) against the oracle restatement."""
    N, n = 256, 10
    c = {"variant": CGGI_BINARY, "N": N, "n": n, "rotation": (16, 4), "trace": (16, 4), "ks": (16, 4)}
    sk = lwe_secret(CGGI_BINARY, n, N, seed=1501)
    z = rlwe_secret(N, seed=1502)
    keys = oracle.sap_keygen(CGGI_BINARY, N, n, (16, 4), (16, 4), (16, 4), 3.2, sk, z, 1503)
    beta = int(np.count_nonzero(sk))
    dec = decomposer(c, keys, beta, 4)
    rng = np.random.default_rng(1504)
    lwes = rng.integers(0, 1 << 12, (2, n + 1), dtype=np.uint64)
    for radix, od in ((2, 13), (N, 3)):
        digits, got = dec.Decompose(lwes, radix, od)
        for j in range(2):
            d, want = oracle.sap_decompose(CGGI_BINARY, N, n, (16, 4), keys[0], (16, 4), keys[1], (16, 4), keys[2],
                                           radix, beta, 4, lwes[j], od)
            assert digits[j] == d
            np.testing.assert_array_equal(got[j], want, err_msg=f"radix {radix} lwe {j}")


def test_batch_order_and_single_calls_agree(native, oracle, cuda):
    c = MANIFEST["bmmp_n256_r8_reset"]
    N, n = c["N"], c["n"]
    sk = lwe_secret(c["variant"], n, N, seed=c["sk_seed"])
    z = rlwe_secret(N, seed=c["sk_seed"] + 1)
    keys = oracle.sap_keygen(c["variant"], N, n, tuple(c["rotation"]), tuple(c["trace"]), tuple(c["ks"]), c["std"],
                             sk, z, c["key_seed"])
    dec = decomposer(c, keys, c["beta"], 3)
    rng = np.random.default_rng(5)
    lwes = rng.integers(0, 1 << 24, (9, n + 1), dtype=np.uint64)
    lwes[4] &= np.uint64(0xFFF)                       # fewer digits, fewer resets
    d_all, all_ = dec.Decompose(lwes, 8, 10)
    d_rev, rev = dec.Decompose(lwes[::-1].copy(), 8, 10)
    np.testing.assert_array_equal(rev[::-1], all_)
    np.testing.assert_array_equal(d_rev[::-1], d_all)
    for j in (0, 4):
        d_one, one = dec.Decompose(lwes[j:j + 1], 8, 10)
        np.testing.assert_array_equal(one[0], all_[j])
        want_d, want = oracle.sap_decompose(c["variant"], N, n, tuple(c["rotation"]), keys[0], tuple(c["trace"]),
                                            keys[1], tuple(c["ks"]), keys[2], 8, c["beta"], 3, lwes[j], 10)
        assert d_one[0] == want_d
        np.testing.assert_array_equal(one[0], want)


def test_decrypts_like_reference_test(native, oracle, cuda):
    """TestDecomp: N = 4096, n = 10, radix 32, noise-free keys, a message mod 32^8 encrypted
    under a binary LWE key; digit i decrypts under the RLWE key to round(2N phase / Q) = m_i."""
    N, n, radix = 4096, 10, 32
    sk = sm64(1401, n) & np.uint64(1)
    z = sm64(1402, N) & np.uint64(1)
    c = {"variant": CGGI_BINARY, "N": N, "n": n, "rotation": (16, 4), "trace": (16, 4), "ks": (16, 4)}
    keys = oracle.sap_keygen(CGGI_BINARY, N, n, (16, 4), (16, 4), (16, 4), 0.0, sk, z, 1403)
    dec = decomposer(c, keys, int(np.count_nonzero(sk)), 2**64 - 1)
    q = radix ** 8
    rng = np.random.default_rng(1404)
    msgs = [int(v) for v in rng.integers(0, q, 4, dtype=np.uint64)]
    lwes = np.zeros((4, n + 1), np.uint64)
    for j, m in enumerate(msgs):
        a = [int(v) for v in rng.integers(0, q, n, dtype=np.uint64)]
        lwes[j, :n] = a
        lwes[j, n] = (sum(x * int(s) for x, s in zip(a, sk)) + m) % q
    digits, got = dec.Decompose(lwes, radix, 9)
    zo = [int(v) for v in z]
    for j, m in enumerate(msgs):
        for i in range(8):
            ct = [int(v) for v in got[j, i]]
            phase = (ct[N] - sum(a * s for a, s in zip(ct[:N], zo))) % P
            assert round(2 * N * phase / P) % (2 * N) == (m >> (5 * i)) % radix, f"lwe {j} digit {i}"


def test_errors(native, cuda):
    from fhetoothpaste_b200 import _native as nat
    L = nat.lib()
    p = nat.BrParams(CGGI_BINARY, nat.GOLDILOCKS, 256, 10, 1 << 16, 4)
    h = ctypes.c_void_p()
    assert L.tp_sap_create(ctypes.byref(p), 1 << 16, 4, 1 << 16, 4, 0, ctypes.byref(h)) == nat.TP_OK
    x = cuda.zeros(11, dtype=cuda.int64, device="cuda")
    y = cuda.zeros(257 * 10, dtype=cuda.int64, device="cuda")
    assert L.tp_sap_decompose_batch(h, 1, y.data_ptr(), 10, x.data_ptr(), 4, 3, 5, None, None) == nat.TP_ERR_STATE
    assert L.tp_sap_key_words(h, 1) == 8 * 4 * 2 * 256 and L.tp_sap_key_words(h, 2) == 256 * 4 * 11
    keys = [np.zeros(L.tp_sap_key_words(h, w), np.uint64) for w in range(3)]
    assert L.tp_sap_upload_keys(h, nat.ptr(keys[0]), keys[0].size, nat.ptr(keys[1]), keys[1].size,
                                nat.ptr(keys[2]), keys[2].size) == nat.TP_OK
    for radix, restart in ((6, 5), (512, 5), (1, 5), (4, 0)):
        assert L.tp_sap_decompose_batch(h, 1, y.data_ptr(), 10, x.data_ptr(), radix, 3, restart, None,
                                        None) == nat.TP_ERR_PARAM
    r = cuda.zeros(2 * 256, dtype=cuda.int64, device="cuda")
    for radix in (1, 3, 512):
        assert L.tp_sap_homtrunc_batch(h, 1, r.data_ptr(), r.data_ptr(), radix, None) == nat.TP_ERR_PARAM
    assert L.tp_sap_reset_batch(h, 1, r.data_ptr(), 6, None) == nat.TP_ERR_PARAM
    x.fill_(1 << 40)                                  # 2^41 needs 21 base-4 digits
    assert L.tp_sap_decompose_batch(h, 1, y.data_ptr(), 10, x.data_ptr(), 4, 3, 5, None, None) == nat.TP_ERR_PARAM
    assert L.tp_sap_destroy(h) == nat.TP_OK
