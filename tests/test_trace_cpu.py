"""TraceEvaluator on the CPU: the oracle (trace steps of tpo_trace_eval, automorphism
evaluation of tpo_auto_eval) against the reference's recorded Eval / EvalAuto outputs
(tests/golden/trace.*)."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import random_acc, rlwe_secret, sha256

GOLD = Path(__file__).resolve().parent / "golden"
MANIFEST = json.loads((GOLD / "trace.json").read_text())


def trace_case(oracle, c):
    keys = oracle.pack_keygen(c["N"], c["basis_log2"], c["digits"], c["std"], rlwe_secret(c["N"], c["sk_seed"]),
                              c["key_seed"])
    return keys, random_acc(c["N"], 2, c["in_seed"])


@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_oracle_trace_matches_reference(oracle, name):
    c = MANIFEST[name]
    N, bl, dg = c["N"], c["basis_log2"], c["digits"]
    keys, x = trace_case(oracle, c)
    assert sha256(keys) == c["key_sha256"] and sha256(x) == c["input_sha256"]
    assert [sha256(oracle.trace_eval(N, bl, dg, keys, x[j])) for j in range(2)] == c["eval_sha256"]
    for t, want in zip(c["auto_index"], c["auto_sha256"]):
        j = (t - 1).bit_length() - 1
        k = keys[(j - 1) * dg * 2 * N:j * dg * 2 * N]
        assert sha256(oracle.auto_eval(N, bl, dg, t, k, x[0])) == want, f"index {t}"
    whole = np.load(GOLD / "trace.npz")
    if name in whole.files:
        np.testing.assert_array_equal(np.stack([oracle.trace_eval(N, bl, dg, keys, x[j]) for j in range(2)]),
                                      whole[name])
