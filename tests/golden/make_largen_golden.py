"""Golden blind rotations at ring sizes above 4096, from the reference library itself.

Run here, where the reference sources exist: `python tests/golden/make_largen_golden.py`
(needs oracle/_ref/libtpref.so, see oracle/Makefile). The reference's SolinasWorker
accepts N up to 2^16; its rotators build a monomial table of N (N + 2) words, so the
cases stop at N = 16384 (2.1 GB). Inputs and keys are regenerated in the tests from the
recorded seeds (same generators as make_golden.py); outputs are recorded as SHA-256 of
each rotation (NTT-domain output, then coefficient output), with the key's SHA-256.
"""
from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests" / "golden"))
from make_golden import br_inputs, case_seed  # noqa: E402
from oracle.oracle import (BMMP_BINARY, CGGI_BINARY, CGGI_TERNARY, Reference, lwe_secret, ptr,  # noqa: E402
                           rlwe_secret, sha256)

OUT = Path(__file__).resolve().parent

# (name, variant, N, n, basis_log2, digits, std)
CASES = [
    ("ternary_n8192", CGGI_TERNARY, 8192, 8, 12, 3, 3.2),
    ("binary_n8192_b16", CGGI_BINARY, 8192, 6, 16, 4, 3.2),
    ("bmmp_n8192", BMMP_BINARY, 8192, 6, 16, 4, 3.2),
    ("ternary_n16384", CGGI_TERNARY, 16384, 4, 12, 3, 3.2),
    ("binary_n16384_l2", CGGI_BINARY, 16384, 4, 20, 2, 3.2),
]


def main() -> None:
    L = Reference().L
    manifest = {"generator": "tests/golden/make_largen_golden.py", "library": "oracle/_ref/libtpref.so", "br": {}}
    for name, variant, N, n, bl, dg, std in CASES:
        t0 = time.time()
        seed = case_seed(name)
        lk = lwe_secret(variant, n, N, seed + 10)
        rk = rlwe_secret(N, seed + 11)
        key_seed = seed + 12
        L.ref_seed(key_seed)
        h = L.ref_br_create(variant, N, n, bl, dg, std, ptr(lk), ptr(rk))
        brk = np.empty(L.ref_br_key_words(h), np.uint64)
        L.ref_br_key_copy(h, ptr(brk))
        lwes, accs, coefs = br_inputs(name, N, n, seed)
        out_sha = []
        for i, oc in enumerate(coefs):
            r = np.empty(2 * N, np.uint64)
            L.ref_br_rotate(h, ptr(r), ptr(np.ascontiguousarray(lwes[i])), ptr(np.ascontiguousarray(accs[i])), oc)
            out_sha.append(sha256(r))
        L.ref_br_destroy(h)
        manifest["br"][name] = {
            "variant": variant, "N": N, "n": n, "basis_log2": bl, "digits": dg, "std": std, "seed": seed,
            "key_seed": key_seed, "key_words": int(brk.size), "key_sha256": sha256(brk),
            "lwe_sha256": sha256(lwes), "acc_sha256": sha256(accs), "out_coef": coefs, "out_sha256": out_sha,
        }
        print(f"{name}: {time.time() - t0:.1f}s", flush=True)
    (OUT / "largen.json").write_text(json.dumps(manifest, indent=1) + "\n")


if __name__ == "__main__":
    main()
