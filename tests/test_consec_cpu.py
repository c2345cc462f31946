"""Consecutive packing on the CPU: the oracle restatement (tpo_pack_consecutive) against the
reference's own PackConsecutively outputs recorded in tests/golden/consec.*, including lengths
that are not powers of two."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import P, rlwe_secret, sha256, uniform_mod

GOLD = Path(__file__).resolve().parent / "golden"
MANIFEST = json.loads((GOLD / "consec.json").read_text())


def consec_case(oracle, c):
    keys = oracle.pack_keygen(c["N"], c["basis_log2"], c["digits"], c["std"], rlwe_secret(c["N"], c["sk_seed"]),
                              c["key_seed"])
    lwes = uniform_mod(c["in_seed"], c["len"] * (c["N"] + 1), P).reshape(c["len"], c["N"] + 1)
    return keys, lwes


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_oracle_consecutive_packing_matches_reference(oracle, name):
    c = MANIFEST[name]
    keys, lwes = consec_case(oracle, c)
    assert sha256(keys) == c["key_sha256"]
    assert sha256(lwes) == c["input_sha256"]
    got = oracle.pack_consecutive(c["N"], c["basis_log2"], c["digits"], keys, lwes, c["len"])
    assert sha256(got) == c["output_sha256"]
    whole = np.load(GOLD / "consec.npz")
    if name in whole.files:
        np.testing.assert_array_equal(got, whole[name])
