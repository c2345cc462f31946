"""Regenerates keys and inputs of the golden key-switching cases."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests" / "golden"))

from make_golden import lwe_ks_secrets  # noqa: E402,F401
from oracle.oracle import P, random_acc, rlwe_secret, sha256, uniform_mod  # noqa: E402

_KEYS: dict = {}


def ks_key(oracle, name: str, c: dict) -> np.ndarray:
    """The case's key in the reference layout, generated by the C oracle (cached)."""
    if name in _KEYS:
        return _KEYS[name]
    N, bl, dg, std, seed = c["N"], c["basis_log2"], c["digits"], c["std"], c["seed"]
    if c["kind"] == "rlwe_ks":
        k = oracle.rlwe_ks_keygen(N, bl, dg, std, rlwe_secret(N, seed + 10), rlwe_secret(N, seed + 11), c["key_seed"])
    elif c["kind"] == "auto":
        k = oracle.auto_keygen(N, bl, dg, std, c["index"], rlwe_secret(N, seed + 10), c["key_seed"])
    elif c["kind"] == "pack":
        k = oracle.pack_keygen(N, bl, dg, std, rlwe_secret(N, seed + 10), c["key_seed"])
    else:
        src, tgt = lwe_ks_secrets(c["n_in"], c["n_out"], seed)
        k = oracle.lwe_ks_keygen(P, c["n_in"], c["n_out"], bl, dg, std, src, tgt, c["key_seed"])
    assert sha256(k) == c["key_sha256"], f"{name}: oracle key generation differs from the reference's"
    _KEYS[name] = k
    return k


def ks_inputs(c: dict) -> np.ndarray:
    seed = c["seed"]
    if c["kind"] in ("rlwe_ks", "auto"):
        x = random_acc(c["N"], 2, seed + 1)
    elif c["kind"] == "pack":
        x = uniform_mod(seed + 1, c["len"] * (c["N"] + 1), P).reshape(c["len"], c["N"] + 1)
    else:
        x = uniform_mod(seed + 1, 2 * (c["n_in"] + 1), P).reshape(2, c["n_in"] + 1)
    assert sha256(x) == c["input_sha256"], "input generator drifted from the golden vectors"
    return x
