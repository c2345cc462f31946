"""LWE -> RGSW scheme switching on the GPU (tp_lwe_to_rgsw_batch): bit-exact against
the reference's recorded outputs (tests/golden/ss.*) and the oracle, batch-order
invariant, and decrypting like the reference's tests/scheme_switch_tests.cpp
(rows of m g_i (-s, 1) for an encrypted bit m)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import (BMMP_BINARY, CGGI_BINARY, P, lwe_encrypt_2n, lwe_inputs, lwe_secret, rlwe_secret,
                           sha256, sm64)

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"
MANIFEST = json.loads((GOLD / "ss.json").read_text())


def converter(c, keys):
    from fhetoothpaste_b200 import GpuLWEtoRGSWConverter
    return GpuLWEtoRGSWConverter((c["variant"], c["N"], c["n"], 1 << c["rotation"][0], c["rotation"][1]),
                                 (1 << c["trace"][0], c["trace"][1]), (1 << c["square"][0], c["square"][1]),
                                 c["out_digits"], 1 << c["out_basis_log2"], *keys)


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_matches_reference_outputs(native, oracle, cuda, name):
    c = MANIFEST[name]
    N, n = c["N"], c["n"]
    sk = lwe_secret(c["variant"], n, N, seed=c["sk_seed"])
    z = rlwe_secret(N, seed=c["sk_seed"] + 1)
    keys = oracle.ss_keygen(c["variant"], N, n, tuple(c["rotation"]), tuple(c["trace"]), tuple(c["square"]),
                            c["std"], sk, z, c["key_seed"])
    assert [sha256(k) for k in keys] == c["key_sha256"]
    conv = converter(c, keys)
    assert sha256(conv.accumulator()) == c["acc_sha256"]
    lwes = lwe_inputs(N, n, c["count"], seed=c["lwe_seed"])
    got = conv.Convert(lwes)
    assert [sha256(g) for g in got] == c["output_sha256"]
    whole = np.load(GOLD / "ss.npz")
    if name in whole.files:
        np.testing.assert_array_equal(got, whole[name])


def test_batch_matches_oracle_and_is_order_invariant(native, oracle, cuda):
    c = {"variant": CGGI_BINARY, "N": 1024, "n": 64, "rotation": (16, 4), "trace": (16, 4), "square": (16, 4),
         "out_digits": 4, "out_basis_log2": 16}
    N, n, batch = c["N"], c["n"], 48
    sk = lwe_secret(CGGI_BINARY, n, N, seed=1201)
    z = rlwe_secret(N, seed=1202)
    keys = oracle.ss_keygen(CGGI_BINARY, N, n, (16, 4), (16, 4), (16, 4), 3.2, sk, z, 1203)
    conv = converter(c, keys)
    lwes = lwe_inputs(N, n, batch, seed=1204)
    got = conv.Convert(lwes)
    for j in (0, 17, batch - 1):
        want = oracle.lwe_to_rgsw(CGGI_BINARY, N, n, (16, 4), keys[0], (16, 4), keys[1], (16, 4), keys[2], 4, 16,
                                  lwes[j])
        np.testing.assert_array_equal(got[j], want, err_msg=f"input {j}")
    rev = conv.Convert(lwes[::-1].copy())
    np.testing.assert_array_equal(rev[::-1], got)
    one = conv.Convert(lwes[5:6])
    np.testing.assert_array_equal(one[0], got[5])


def phases(oracle, out, z, N, rows):
    zn = oracle.ntt_forward(z).astype(object)
    res = []
    for i in range(rows):
        A = out[i * 2 * N:i * 2 * N + N].astype(object)
        B = out[i * 2 * N + N:(i + 1) * 2 * N].astype(object)
        res.append(oracle.ntt_backward(np.array((B - A * zn) % P, dtype=np.uint64)))
    return res


@pytest.mark.parametrize("variant,D,beta", [(CGGI_BINARY, 4, 16), (BMMP_BINARY, 4, 10)],
                         ids=["cggi_exact_digits", "bmmp_approx_digits"])
def test_decrypts_like_reference_test(native, oracle, cuda, variant, D, beta):
    """scheme_switch_tests.cpp TestConvExactDigs / TestConvApproxDigs at N = 2048, n = 100,
    noise-free keys and a binary RLWE key: row i of lev_right has phase m 2^(beta (max - D + i))
    and row i of lev_left -s times it, max = ceil(64 / beta)."""
    c = {"variant": variant, "N": 2048, "n": 100, "rotation": (16, 4), "trace": (16, 4), "square": (16, 4),
         "out_digits": D, "out_basis_log2": beta}
    N, n = 2048, 100
    sk = lwe_secret(variant, n, N, seed=1301)
    z = sm64(1302, N) & np.uint64(1)
    keys = oracle.ss_keygen(variant, N, n, (16, 4), (16, 4), (16, 4), 0.0, sk, z, 1303)
    conv = converter(c, keys)
    msgs = [0, 1, 1, 0, 1, 0, 0, 1]
    lwes = lwe_encrypt_2n(sk, N, [m * N for m in msgs], seed=1304)
    got = conv.Convert(lwes)
    shift = -(-64 // beta) - D
    zo = z.astype(object)
    for j, m in enumerate(msgs):
        ph = phases(oracle, got[j], z, N, 2 * D)
        for i in range(D):
            scal = (m << (beta * (shift + i))) % P
            left = np.array((P - scal) * zo % P, dtype=np.uint64)
            right = np.zeros(N, np.uint64)
            right[0] = scal
            np.testing.assert_array_equal(ph[i], left, err_msg=f"lwe {j} left row {i}")
            np.testing.assert_array_equal(ph[D + i], right, err_msg=f"lwe {j} right row {i}")


def test_errors(native, oracle, cuda):
    import ctypes
    from fhetoothpaste_b200 import _native as nat
    L = nat.lib()
    p = nat.BrParams(CGGI_BINARY, nat.GOLDILOCKS, 256, 16, 1 << 16, 4)
    h = ctypes.c_void_p()
    # out_digits must split N into even blocks; the first scale must fit an int shift
    assert L.tp_ss_create(ctypes.byref(p), 1 << 16, 4, 1 << 16, 4, 3, 1 << 16, 0, ctypes.byref(h)) == nat.TP_ERR_PARAM
    assert L.tp_ss_create(ctypes.byref(p), 1 << 16, 4, 1 << 16, 4, 2, 1 << 16, 0, ctypes.byref(h)) == nat.TP_ERR_PARAM
    assert L.tp_ss_create(ctypes.byref(p), 1 << 16, 4, 1 << 16, 4, 4, 1 << 16, 0, ctypes.byref(h)) == nat.TP_OK
    x = cuda.zeros(17, dtype=cuda.int64, device="cuda")
    y = cuda.zeros(4 * 256 * 4, dtype=cuda.int64, device="cuda")
    assert L.tp_lwe_to_rgsw_batch(h, 1, y.data_ptr(), x.data_ptr(), None) == nat.TP_ERR_STATE
    assert L.tp_ss_key_words(h, 0) == oracle.L.tpo_brk_words(CGGI_BINARY, 256, 16, 4)
    assert L.tp_ss_key_words(h, 1) == 8 * 4 * 2 * 256 and L.tp_ss_key_words(h, 2) == 4 * 2 * 256
    assert L.tp_ss_upload_keys(h, None, 0, None, 0, None, 0) != nat.TP_OK
    assert L.tp_ss_destroy(h) == nat.TP_OK
