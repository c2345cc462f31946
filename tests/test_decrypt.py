"""Decryption invariants of the blind rotation, restated from the reference's tests.

* tests/cggi_blind_rotation_test.cpp:95-123: with noise-free keys and an exact gadget
  (base 2^16, l = 4), the phase of BlindRotate(lwe(msg), RLWE(data)) equals data * X^msg
  word for word (data = [0, 1, .., N-1 | -0, -1, ..]).
* With Gaussian noise (sigma = 3.2) the phase is within the noise bound of the rotated
  test polynomial, so a LUT value encoded at Delta = p/16 decodes exactly.
* Base 2^12, l = 3 (ternary / BMMP configs): the reference's keys scale RGSW row j by
  2^(60-12j) while the signed decomposition weights digit j by 2^(52-12j)
  (lib/include/static/gadget_decomp.h:176 vs lib/src/base_crypto.cpp:68,85-95), so the
  reference's own output does not decrypt; a key with rows aligned to the digits
  (oracle `br_keygen_aligned`) rotates through the same kernels and decrypts.

The CPU tests run the oracle at small sizes; the GPU tests rotate full-size configs on
the device, compare with the oracle word for word, then decrypt.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle.oracle import (BMMP_BINARY, CGGI_BINARY, CGGI_TERNARY, P, lwe_encrypt_2n, lwe_secret, rlwe_secret,
                           sm64, uniform_mod)

DELTA = P // 16


def rotate_poly(f: np.ndarray, k: int) -> np.ndarray:
    """f * X^k in Z_p[X]/(X^N + 1), 0 <= k < 2N."""
    N = f.size
    neg = lambda v: np.where(v == 0, v, np.uint64(P) - v)  # noqa: E731
    if k >= N:
        return neg(rotate_poly(f, k - N))
    out = np.empty_like(f)
    out[k:] = f[:N - k]
    out[:k] = neg(f[N - k:])
    return out


def centered_error(got: np.ndarray, want: np.ndarray) -> int:
    d = [(int(a) - int(b)) % P for a, b in zip(got, want)]
    return max(min(x, P - x) for x in d)


def coef_acc(oracle, N, std, msg, sk, seed):
    """RLWE encryption of msg moved to the coefficient domain, as the reference test builds it."""
    ct = oracle.make_rlwe(N, std, msg, sk, seed)
    return np.concatenate([oracle.ntt_backward(ct[:N]), oracle.ntt_backward(ct[N:])])


def lut_poly(N: int, table) -> np.ndarray:
    """Test polynomial with table[k] * Delta on the k-th run of N/16 coefficients."""
    per = N // len(table)
    return np.array([(int(table[i // per]) * DELTA) % P for i in range(N)], dtype=np.uint64)


# ---------------------------------------------------------------------------
# CPU: the oracle at small sizes
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("variant", [CGGI_BINARY, CGGI_TERNARY, BMMP_BINARY], ids=["binary", "ternary", "bmmp"])
def test_exact_rotation_invariant(oracle, variant):
    N, n = 256, 10
    lk = lwe_secret(variant, n, N, seed=101)
    rk = uniform_mod(102, N, P)  # the reference test draws the RLWE key uniformly mod Q
    brk = oracle.br_keygen(variant, N, n, 16, 4, 0.0, lk, rk, seed=103)
    data = np.array([i for i in range(N)], dtype=np.uint64)
    acc = coef_acc(oracle, N, 0.0, data, rk, seed=104)
    for t, msg in enumerate(N + sm64(105, 3) % np.uint64(N)):
        lwe = lwe_encrypt_2n(lk, N, [int(msg)], seed=106 + t)[0]
        res = oracle.blind_rotate(variant, N, n, 16, 4, brk, lwe, acc, False)
        phase = oracle.phase_rlwe(res, rk)
        np.testing.assert_array_equal(phase, rotate_poly(data, int(msg)))


@pytest.mark.parametrize("variant,beta,digits", [(CGGI_BINARY, 16, 4), (CGGI_TERNARY, 16, 4), (BMMP_BINARY, 16, 4),
                                                 (CGGI_BINARY, 12, 3)],
                         ids=["binary_b16", "ternary_b16", "bmmp_b16", "binary_b12"])
def test_lut_decrypts_with_noise(oracle, variant, beta, digits):
    N, n = 512, 16
    lk = lwe_secret(variant, n, N, seed=111)
    rk = rlwe_secret(N, seed=112)
    brk = oracle.br_keygen(variant, N, n, beta, digits, 3.2, lk, rk, seed=113)
    table = sm64(114, 16) % np.uint64(16)
    f = lut_poly(N, table)
    acc = np.concatenate([np.zeros(N, np.uint64), f])
    msgs = [int(m) * (2 * N // 16) for m in sm64(115, 4) % np.uint64(8)]
    lwes = lwe_encrypt_2n(lk, N, msgs, seed=116)
    for lwe, msg in zip(lwes, msgs):
        phase = oracle.phase_rlwe(oracle.blind_rotate(variant, N, n, beta, digits, brk, lwe, acc, False), rk)
        assert centered_error(phase, rotate_poly(f, msg)) < 2**50


@pytest.mark.parametrize("variant", [CGGI_TERNARY, BMMP_BINARY], ids=["ternary", "bmmp"])
def test_base_2_12_needs_aligned_gadget(oracle, variant):
    N, n = 512, 16
    lk = lwe_secret(variant, n, N, seed=121)
    rk = rlwe_secret(N, seed=122)
    f = lut_poly(N, sm64(123, 16) % np.uint64(16))
    acc = np.concatenate([np.zeros(N, np.uint64), f])
    msg = 3 * (2 * N // 16)
    lwe = lwe_encrypt_2n(lk, N, [msg], seed=124)[0]
    ref_key = oracle.br_keygen(variant, N, n, 12, 3, 3.2, lk, rk, seed=125)
    aligned = oracle.br_keygen_aligned(variant, N, n, 12, 3, 3.2, lk, rk, seed=125)
    want = rotate_poly(f, msg)
    err_ref = centered_error(oracle.phase_rlwe(oracle.blind_rotate(variant, N, n, 12, 3, ref_key, lwe, acc, False),
                                               rk), want)
    err_aligned = centered_error(
        oracle.phase_rlwe(oracle.blind_rotate(variant, N, n, 12, 3, aligned, lwe, acc, False), rk), want)
    assert err_ref > DELTA // 2, "reference keys at base 2^12, l = 3 unexpectedly decrypt"
    assert err_aligned < 2**50


def test_aligned_key_equals_reference_key_when_beta_divides_64(oracle):
    N, n = 128, 4
    lk = lwe_secret(CGGI_BINARY, n, N, seed=131)
    rk = rlwe_secret(N, seed=132)
    a = oracle.br_keygen(CGGI_BINARY, N, n, 16, 4, 3.2, lk, rk, seed=133)
    b = oracle.br_keygen_aligned(CGGI_BINARY, N, n, 16, 4, 3.2, lk, rk, seed=133)
    np.testing.assert_array_equal(a, b)


# ---------------------------------------------------------------------------
# GPU: full-size configs
# ---------------------------------------------------------------------------

GPU_CONFIGS = [  # (name, variant, N, n, beta, digits, aligned key)
    ("cfg1_binary_n1024_b16", CGGI_BINARY, 1024, 500, 16, 4, False),
    ("cfg2_ternary_n2048_b12_aligned", CGGI_TERNARY, 2048, 630, 12, 3, True),
    ("cfg3_bmmp_n2048_b16", BMMP_BINARY, 2048, 768, 16, 4, False),
]


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", GPU_CONFIGS, ids=[c[0] for c in GPU_CONFIGS])
def test_gpu_lut_decrypts_at_full_size(native, oracle, cuda, cfg):
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    _, variant, N, n, beta, digits, aligned = cfg
    lk = lwe_secret(variant, n, N, seed=141)
    rk = rlwe_secret(N, seed=142)
    keygen = oracle.br_keygen_aligned if aligned else oracle.br_keygen
    brk = keygen(variant, N, n, beta, digits, 3.2, lk, rk, seed=143)
    rot = GpuBlindRotator(BlindRotationContext(variant, N, n, 1 << beta, digits), brk)
    count = 8
    tables = sm64(144, 16 * count).reshape(count, 16) % np.uint64(16)
    fs = np.stack([lut_poly(N, t) for t in tables])
    accs = np.concatenate([np.zeros((count, N), np.uint64), fs], axis=1)
    msgs = [int(m) * (2 * N // 16) for m in sm64(145, count) % np.uint64(16)]
    lwes = lwe_encrypt_2n(lk, N, msgs, seed=146)
    got = rot.blind_rotate_batch_host(lwes, accs, out_coef=False)
    want = oracle.blind_rotate_many(variant, N, n, beta, digits, brk, lwes, accs, False, 8)
    np.testing.assert_array_equal(got, want)
    for i in range(count):
        phase = oracle.phase_rlwe(got[i], rk)
        assert centered_error(phase, rotate_poly(fs[i], msgs[i])) < 2**52
        # coefficient 0 decodes to the LUT entry the message selects
        decoded = (int(phase[0]) + DELTA // 2) % P // DELTA
        assert decoded == int(rotate_poly(fs[i], msgs[i])[0]) // DELTA
