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


def integer_switch(v: int, k: int, kind: str) -> int:
    """The GPU kernel's integer form of the long-double switch (ms_pow2 in ks_util_kernels.cuh):
    v 2^k = a p + r; x = a + F 2^-s in a's binade, s = 64 - bitlength(a) (65 when a = 0)."""
    hi, lo = v >> (64 - k), (v << k) & (2**64 - 1)
    t = lo + hi * (2**32 - 1)
    a, r = (hi + 1, t - P) if t >= P else (hi, t)
    res = a
    if r and kind != "floor":
        s = 64 - a.bit_length() if a else 65
        if kind == "ceil":
            res = a if (a and r <= (P >> (s + 1))) else a + 1
        else:
            tail = P >> s if s < 64 else 0
            res = a + 1 if r >= (P - tail + 1) // 2 else a
    return res - (1 << k) if res >= (1 << k) else res


def test_integer_form_equals_long_double_switch(oracle):
    """The integer form against the oracle's 80-bit long double on random words (some >= p), and the
    neighbours of every rounding boundary m p / 2^k and (m + 1/2) p / 2^k, k from 1 to 32."""
    rng = np.random.default_rng(11)
    for k in (1, 2, 7, 11, 12, 13, 20, 31, 32):
        T = 1 << k
        xs = [int(v) for v in rng.integers(0, 2**64 - 1, 1500, dtype=np.uint64)] + [0, 1, P - 1, P, P + 1, 2**64 - 1]
        for m in np.linspace(0, T - 1, 120).astype(np.int64).tolist():
            for base in ((m * P) // T, ((2 * m + 1) * P) // (2 * T)):
                xs += [base + d for d in range(-3, 4) if 0 <= base + d < 2**64]
        arr = np.array(xs, dtype=np.uint64)
        for kind in ("round", "floor", "ceil"):
            want = oracle.modulus_switch(arr, P, T, kind)
            got = np.array([integer_switch(x, k, kind) for x in xs], dtype=np.uint64)
            np.testing.assert_array_equal(got, want, err_msg=f"{kind} to 2^{k}")
