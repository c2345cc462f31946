"""Golden vectors for SAP digit decomposition (SAPDecomposer::Decompose, HomTrunc,
ResetAccumulator; lib/src/operators/sap_decomposer.cpp) from the reference library
built in oracle/_ref. Run in the container that has the reference build:

    python tests/golden/make_sap_golden.py

Keys are made by the reference (SAPDecompositionContext::ConstructOperator) from
the shimmed sampler seeded with `key_seed`; the record holds their SHA-256 and the
oracle regenerates them from the same seed. Inputs are regenerated from their
seeds and checked against the recorded hash. The reference's variance model puts
the restart period at UINT64_MAX for every context here (its trace variance is 0),
so resets are forced by setting the operator's period (cases with `restart`); each
case keeps to one reset per decomposition, because the reference's LWE converter
clears only part of its accumulator between calls (lwe_conversion.cpp:217). Every
decomposition runs on a converter whose accumulator is cleared first. Radix >= 4
and N >= 256: below those the reference's HomTrunc overruns its buffer or crashes.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle.oracle import (BMMP_BINARY, CGGI_BINARY, CGGI_TERNARY, Reference, lwe_secret, ptr,  # noqa: E402
                           random_acc, rlwe_secret, sha256)

OUT = Path(__file__).resolve().parent

# name, variant, N, n, rotation, trace, ks (basis_log2, digits), std, radix, input bits,
# inputs, restart (None: the context's), store whole outputs
CASES = [
    ("binary_n256_r4", CGGI_BINARY, 256, 10, (16, 4), (16, 4), (16, 4), 3.2, 4, 16, 3, None, True),
    ("binary_n256_r4_reset", CGGI_BINARY, 256, 10, (16, 4), (16, 4), (16, 4), 3.2, 4, 16, 2, 5, True),
    ("bmmp_n256_r8_reset", BMMP_BINARY, 256, 10, (16, 4), (14, 4), (12, 5), 3.2, 8, 24, 2, 5, True),
    ("ternary_n256_r4", CGGI_TERNARY, 256, 10, (12, 3), (16, 4), (16, 4), 3.2, 4, 9, 2, None, True),
    ("binary_n1024_r32", CGGI_BINARY, 1024, 10, (16, 4), (16, 4), (16, 4), 3.2, 32, 40, 1, None, True),
    ("binary_n4096_r32", CGGI_BINARY, 4096, 10, (16, 4), (16, 4), (16, 4), 0.0, 32, 40, 1, None, False),
]


def case_inputs(n: int, bits: int, count: int, seed: int) -> np.ndarray:
    """count x (n+1) words below 2^bits; the second LWE (if any) has words below 2^(bits/2), so a
    batch mixes digit counts, and the third starts with a_0 = 0."""
    rng = np.random.default_rng(seed)
    x = rng.integers(0, 1 << bits, (count, n + 1), dtype=np.uint64)
    if count > 1:
        x[1] &= np.uint64((1 << (bits // 2)) - 1)
    if count > 2:
        x[2, 0] = 0
    return x


def digits_for(N: int, radix: int, bits: int) -> int:
    r = radix.bit_length() - 1
    return -(-bits // r) + 1


def main() -> None:
    L = Reference().L
    manifest, arrays = {}, {}
    for i, (name, variant, N, n, br, tr, ks, std, radix, bits, count, restart, whole) in enumerate(CASES):
        key_seed, in_seed, sk_seed = 700 + i, 750 + i, 780 + i
        sk = lwe_secret(variant, n, N, seed=sk_seed)
        z = rlwe_secret(N, seed=sk_seed + 1)
        L.ref_seed(key_seed)
        h = L.ref_sap_create(variant, N, n, br[0], br[1], tr[0], tr[1], ks[0], ks[1], std, radix, ptr(sk), ptr(z))
        if restart is not None:
            L.ref_sap_set_restart(h, restart)
        key_sha = []
        for w in range(3):
            k = np.empty(L.ref_sap_key_words(h, w), np.uint64)
            L.ref_sap_key_copy(h, w, ptr(k))
            key_sha.append(sha256(k))
        lwes = case_inputs(n, bits, count, in_seed)
        od = digits_for(N, radix, bits)
        outs = np.zeros((count, od, N + 1), np.uint64)
        for j in range(count):
            L.ref_sap_decompose(h, ptr(outs[j]), outs[j].size, ptr(lwes[j]), radix)
        rec = {"variant": variant, "N": N, "n": n, "rotation": list(br), "trace": list(tr), "ks": list(ks),
               "std": std, "radix": radix, "bits": bits, "count": count, "out_digits": od,
               "restart": int(L.ref_sap_restart(h)), "beta": int(L.ref_sap_beta(h)), "key_seed": key_seed,
               "in_seed": in_seed, "sk_seed": sk_seed, "key_sha256": key_sha, "input_sha256": sha256(lwes),
               "output_sha256": [sha256(o) for o in outs]}
        if N <= 1024:
            # HomTrunc and ResetAccumulator on one random NTT-domain RLWE each
            x = random_acc(N, 2, in_seed + 1)
            ht = np.empty(2 * N, np.uint64)
            L.ref_sap_homtrunc(h, ptr(ht), ptr(x[0].copy()), radix)
            rs = x[1].copy()
            L.ref_sap_reset(h, ptr(rs), 0)
            rec["homtrunc_sha256"] = sha256(ht)
            rec["reset_sha256"] = sha256(rs)
        L.ref_sap_destroy(h)
        manifest[name] = rec
        if whole:
            arrays[name] = outs
        print(name, "done", flush=True)
    np.savez_compressed(OUT / "sap.npz", **arrays)
    (OUT / "sap.json").write_text(json.dumps(manifest, indent=1) + "\n")
    print("wrote", OUT / "sap.npz")


if __name__ == "__main__":
    main()
