"""Regenerates the inputs and keys of the golden blind-rotation cases."""
from __future__ import annotations

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests" / "golden"))

from make_golden import br_inputs  # noqa: E402
from oracle.oracle import lwe_secret, rlwe_secret, sha256  # noqa: E402

_KEYS: dict = {}


def case_key(oracle, name: str, case: dict):
    """(lwe_key, rlwe_key, brk) of a golden case, brk made by the C oracle (cached)."""
    if name not in _KEYS:
        N, n, v = case["N"], case["n"], case["variant"]
        lk = lwe_secret(v, n, N, case["seed"] + 10)
        rk = rlwe_secret(N, case["seed"] + 11)
        brk = oracle.br_keygen(v, N, n, case["basis_log2"], case["digits"], case["std"], lk, rk, case["key_seed"])
        _KEYS[name] = (lk, rk, brk)
    return _KEYS[name]


def case_inputs(name: str, case: dict):
    lwes, accs, coefs = br_inputs(name, case["N"], case["n"], case["seed"])
    assert sha256(lwes) == case["lwe_sha256"], "LWE input generator drifted from the golden vectors"
    assert sha256(accs) == case["acc_sha256"], "accumulator generator drifted from the golden vectors"
    return lwes, accs, coefs
