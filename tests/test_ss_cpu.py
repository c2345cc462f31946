"""LWE -> RGSW scheme switching on the CPU: the oracle restatement
(oracle/tp_oracle.c, tpo_ss_*) against the reference's own outputs recorded in
tests/golden/ss.* (LWEtoRGSWConverter::Convert, lib/src/operators/
lwe_to_rgsw_conversion.cpp:168-225): the keys the reference makes from a
sampler seed, its test polynomial and its RGSW outputs, bit for bit."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import lwe_inputs, lwe_secret, rlwe_secret, sha256

GOLD = Path(__file__).resolve().parent / "golden"
MANIFEST = json.loads((GOLD / "ss.json").read_text())


def case_inputs(oracle, c):
    N, n, v = c["N"], c["n"], c["variant"]
    sk = lwe_secret(v, n, N, seed=c["sk_seed"])
    z = rlwe_secret(N, seed=c["sk_seed"] + 1)
    keys = oracle.ss_keygen(v, N, n, tuple(c["rotation"]), tuple(c["trace"]), tuple(c["square"]), c["std"], sk, z,
                            c["key_seed"])
    lwes = lwe_inputs(N, n, c["count"], seed=c["lwe_seed"])
    return keys, lwes


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_oracle_keys_and_test_polynomial_match_reference(oracle, name):
    c = MANIFEST[name]
    keys, lwes = case_inputs(oracle, c)
    assert [sha256(k) for k in keys] == c["key_sha256"]
    assert sha256(lwes) == c["input_sha256"]
    assert sha256(oracle.ss_test_poly(c["N"], c["out_digits"], c["out_basis_log2"])) == c["acc_sha256"]


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_oracle_conversion_matches_reference(oracle, name):
    c = MANIFEST[name]
    (brk, trk, sqk), lwes = case_inputs(oracle, c)
    whole = np.load(GOLD / "ss.npz")
    for j in range(c["count"]):
        got = oracle.lwe_to_rgsw(c["variant"], c["N"], c["n"], tuple(c["rotation"]), brk, tuple(c["trace"]), trk,
                                 tuple(c["square"]), sqk, c["out_digits"], c["out_basis_log2"], lwes[j])
        assert sha256(got) == c["output_sha256"][j], f"{name} input {j}"
        if name in whole.files:
            np.testing.assert_array_equal(got, whole[name][j])


def test_test_polynomial_layout(oracle):
    """Block 0 holds +-scale/2 around X^0 with the sign of -tp, block b >= 1 scale 2^(b beta) / 2."""
    from oracle.oracle import P
    N, D, beta = 256, 4, 16
    acc = oracle.ss_test_poly(N, D, beta).astype(object)
    bs = N // D
    half = (P + 1) // 2
    tp = acc[2 * N:]
    assert all(v == 0 for v in acc[:N])
    assert all((a + b) % P == 0 for a, b in zip(acc[N:2 * N], tp))
    assert tp[0] == half and tp[N - 1] == P - half
    for b in range(1, D):
        assert tp[b * bs] == (1 << (beta * b)) * half % P


@pytest.mark.parametrize("D,beta", [(2, 16), (1, 16), (4, 7)])
def test_test_polynomial_rejects_overflowing_first_scale(oracle, D, beta):
    """The reference's first scale is the int shift 1 << beta (max_digits - D); from 31 on it overflows."""
    from oracle.oracle import ptr
    acc = np.empty(3 * 256, np.uint64)
    assert oracle.L.tpo_ss_test_poly(256, D, beta, ptr(acc)) == -1
