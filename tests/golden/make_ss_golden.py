"""Golden vectors for LWE -> RGSW scheme switching (LWEtoRGSWConverter::Convert,
lib/src/operators/lwe_to_rgsw_conversion.cpp:168-225) from the reference library
built in oracle/_ref. Run in the container that has the reference build:

    python tests/golden/make_ss_golden.py

Keys are made by the reference (SchemeSwitchingContext::ConstructOperator) from
the shimmed sampler seeded with `key_seed`; the record holds their SHA-256, and
the oracle regenerates them from the same seed. Inputs are regenerated from
their seeds and checked against the recorded input hash. Outputs are stored
whole for the small rings and as SHA-256 for N = 2048 (the shapes of the
reference's tests/scheme_switch_tests.cpp, on the Goldilocks modulus).
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle.oracle import (BMMP_BINARY, CGGI_BINARY, CGGI_TERNARY, Reference, lwe_inputs, lwe_secret,  # noqa: E402
                           ptr, rlwe_secret, sha256)

OUT = Path(__file__).resolve().parent

# name, variant, N, n, rotation (basis_log2, digits), trace gadget, squaring gadget, std,
# out_digits, out_basis_log2, inputs, store whole outputs
CASES = [
    ("binary_n256", CGGI_BINARY, 256, 16, (16, 4), (16, 4), (16, 4), 3.2, 4, 16, 2, True),
    ("bmmp_mixed_n256", BMMP_BINARY, 256, 16, (12, 5), (14, 4), (20, 3), 3.2, 4, 10, 2, True),
    ("ternary_n128", CGGI_TERNARY, 128, 10, (16, 4), (14, 5), (16, 4), 3.2, 2, 30, 2, True),
    ("binary_n2048_b14", CGGI_BINARY, 2048, 100, (14, 4), (14, 4), (14, 4), 3.2, 4, 14, 1, False),
    ("bmmp_n2048_approx", BMMP_BINARY, 2048, 100, (14, 4), (14, 4), (14, 4), 3.2, 4, 10, 1, False),
]


def main() -> None:
    ref = Reference()
    L = ref.L
    manifest, arrays = {}, {}
    for i, (name, variant, N, n, br, tr, sq, std, D, ob, count, whole) in enumerate(CASES):
        key_seed, lwe_seed, sk_seed = 900 + i, 950 + i, 980 + i
        sk = lwe_secret(variant, n, N, seed=sk_seed)
        z = rlwe_secret(N, seed=sk_seed + 1)
        L.ref_seed(key_seed)
        h = L.ref_ss_create(variant, N, n, br[0], br[1], tr[0], tr[1], sq[0], sq[1], std, D, ob, ptr(sk), ptr(z))
        key_sha = []
        for w in range(3):
            k = np.empty(L.ref_ss_key_words(h, w), np.uint64)
            L.ref_ss_key_copy(h, w, ptr(k))
            key_sha.append(sha256(k))
        acc = np.empty(3 * N, np.uint64)
        L.ref_ss_test_poly(h, ptr(acc))
        lwes = lwe_inputs(N, n, count, seed=lwe_seed)
        outs = np.empty((count, 4 * N * D), np.uint64)
        for j in range(count):
            L.ref_ss_convert(h, ptr(outs[j]), ptr(lwes[j]))
        L.ref_ss_destroy(h)
        manifest[name] = {"variant": variant, "N": N, "n": n, "rotation": list(br), "trace": list(tr),
                          "square": list(sq), "std": std, "out_digits": D, "out_basis_log2": ob, "count": count,
                          "key_seed": key_seed, "lwe_seed": lwe_seed, "sk_seed": sk_seed,
                          "key_sha256": key_sha, "input_sha256": sha256(lwes), "acc_sha256": sha256(acc),
                          "output_sha256": [sha256(o) for o in outs]}
        if whole:
            arrays[name] = outs
        print(name, "done", flush=True)
    np.savez_compressed(OUT / "ss.npz", **arrays)
    (OUT / "ss.json").write_text(json.dumps(manifest, indent=1) + "\n")
    print("wrote", OUT / "ss.npz")


if __name__ == "__main__":
    main()
