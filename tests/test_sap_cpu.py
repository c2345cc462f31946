"""SAP digit decomposition on the CPU: the oracle restatement (oracle/tp_oracle.c,
tpo_sap_*) against the reference's own outputs recorded in tests/golden/sap.*
(SAPDecomposer::Decompose / HomTrunc / ResetAccumulator, lib/src/operators/
sap_decomposer.cpp): keys from the sampler seed, the decomposition digits with and
without an accumulator reset, for CGGI binary / ternary and BMMP rotators."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import lwe_secret, random_acc, rlwe_secret, sha256

GOLD = Path(__file__).resolve().parent / "golden"
sys.path.insert(0, str(GOLD))
from make_sap_golden import case_inputs  # noqa: E402

MANIFEST = json.loads((GOLD / "sap.json").read_text())
SMALL = sorted(k for k, c in MANIFEST.items() if c["N"] <= 1024)


def case_keys(oracle, c):
    sk = lwe_secret(c["variant"], c["n"], c["N"], seed=c["sk_seed"])
    z = rlwe_secret(c["N"], seed=c["sk_seed"] + 1)
    return oracle.sap_keygen(c["variant"], c["N"], c["n"], tuple(c["rotation"]), tuple(c["trace"]), tuple(c["ks"]),
                             c["std"], sk, z, c["key_seed"]), sk


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_keys_inputs_and_weight_match_reference(oracle, name):
    c = MANIFEST[name]
    keys, sk = case_keys(oracle, c)
    assert [sha256(k) for k in keys] == c["key_sha256"]
    assert sha256(case_inputs(c["n"], c["bits"], c["count"], c["in_seed"])) == c["input_sha256"]
    assert int(np.count_nonzero(sk)) == c["beta"]


@pytest.mark.parametrize("name", SMALL)
def test_oracle_decomposition_matches_reference(oracle, name):
    c = MANIFEST[name]
    (brk, trk, ksk), _ = case_keys(oracle, c)
    lwes = case_inputs(c["n"], c["bits"], c["count"], c["in_seed"])
    whole = np.load(GOLD / "sap.npz")
    for j in range(c["count"]):
        _, got = oracle.sap_decompose(c["variant"], c["N"], c["n"], tuple(c["rotation"]), brk, tuple(c["trace"]),
                                      trk, tuple(c["ks"]), ksk, c["radix"], c["beta"], c["restart"], lwes[j],
                                      c["out_digits"])
        assert sha256(got) == c["output_sha256"][j], f"{name} input {j}"
        np.testing.assert_array_equal(got, whole[name][j])


@pytest.mark.parametrize("name", SMALL)
def test_oracle_homtrunc_and_reset_match_reference(oracle, name):
    c = MANIFEST[name]
    (brk, trk, ksk), _ = case_keys(oracle, c)
    x = random_acc(c["N"], 2, c["in_seed"] + 1)
    assert sha256(oracle.sap_homtrunc(c["N"], tuple(c["trace"]), trk, c["radix"], x[0])) == c["homtrunc_sha256"]
    got = oracle.sap_reset(c["variant"], c["N"], c["n"], tuple(c["rotation"]), brk, tuple(c["ks"]), ksk, 0, x[1])
    assert sha256(got) == c["reset_sha256"]


def test_input_modulus_rule(oracle):
    """2^IntLog2(a_0), doubled once for every later word it does not exceed (sap_decomposer.cpp:409-416)."""
    L = oracle.L
    assert [L.tpo_ref_int_log2(x) for x in (0, 1, 2, 3, 4, 5, 1 << 40, (1 << 40) + 1)] == [0, 0, 1, 2, 2, 3, 40, 41]
