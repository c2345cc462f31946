"""ModulusSwitch (lib/src/static/modulus_switching.cpp:36-93): the oracle against golden vectors
taken from the reference build (tests/golden/make_modswitch_golden.py), on boundary inputs."""
import json
from pathlib import Path

import numpy as np

from oracle.oracle import P, sha256

GOLD = Path(__file__).resolve().parent / "golden"


def test_oracle_matches_reference_golden(oracle):
    manifest = json.loads((GOLD / "modswitch.json").read_text())
    d = np.load(GOLD / "modswitch.npz")
    for t, meta in manifest.items():
        x = d[f"in_{t}"]
        assert sha256(x) == meta["input_sha256"]
        for kind in ("round", "floor", "ceil"):
            np.testing.assert_array_equal(oracle.modulus_switch(x, P, int(t), kind), d[f"{kind}_{t}"],
                                          err_msg=f"{kind} to {t}")


def test_floor_to_power_of_two_is_exact_integer_floor():
    """p = 1 (mod 2^k) keeps every quotient v 2^k / p more than half a long-double ulp below the next
    integer, so the reference's floorl equals the exact floor (what the GPU kernel computes)."""
    d = np.load(GOLD / "modswitch.npz")
    for t in (256, 2048, 4096, 8192):
        x = d[f"in_{t}"]
        exact = np.array([(int(v) * t) // P for v in x], dtype=np.uint64)
        np.testing.assert_array_equal(d[f"floor_{t}"], exact)
