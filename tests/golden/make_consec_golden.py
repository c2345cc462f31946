"""Golden vectors for consecutive packing (LWEtoRLWEPacker::PackConsecutively,
lib/src/operators/lwe_to_rlwe_packing.cpp:260-393) from the reference library built in
oracle/_ref. Run in the container that has the reference build:

    python tests/golden/make_consec_golden.py

The packer's automorphism keys come from the shimmed sampler seeded with `key_seed`
(their SHA-256 is recorded; the oracle regenerates them from the same seed); inputs
are uniform words mod p regenerated from `in_seed`. Lengths include non-powers of two.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle.oracle import P, Reference, ptr, rlwe_secret, sha256, uniform_mod  # noqa: E402

OUT = Path(__file__).resolve().parent

# name, N, basis_log2, digits, len, store the output whole
CASES = [
    ("consec2_n256", 256, 16, 4, 2, True),
    ("consec7_n256", 256, 16, 4, 7, True),
    ("consec64_n256", 256, 16, 4, 64, True),
    ("consec100_n256", 256, 16, 4, 100, True),
    ("consec256_n256", 256, 16, 4, 256, True),
    ("consec5_n128_b12", 128, 12, 3, 5, True),
    ("consec64_n2048", 2048, 16, 4, 64, False),
]


def main() -> None:
    L = Reference().L
    manifest, arrays = {}, {}
    for i, (name, N, bl, dg, length, whole) in enumerate(CASES):
        key_seed, in_seed, sk_seed = 600 + i, 630 + i, 660 + i
        key = rlwe_secret(N, sk_seed)
        L.ref_seed(key_seed)
        h = L.ref_pack_create(N, bl, dg, 3.2, ptr(key))
        keys = np.empty((N.bit_length() - 1) * dg * 2 * N, np.uint64)
        L.ref_pack_key_copy(h, ptr(keys))
        lwes = uniform_mod(in_seed, length * (N + 1), P).reshape(length, N + 1)
        out = np.empty(2 * N, np.uint64)
        L.ref_pack_consecutive(h, ptr(out), ptr(lwes), length)
        L.ref_pack_destroy(h)
        manifest[name] = {"N": N, "basis_log2": bl, "digits": dg, "std": 3.2, "len": length, "key_seed": key_seed,
                          "in_seed": in_seed, "sk_seed": sk_seed, "key_sha256": sha256(keys),
                          "input_sha256": sha256(lwes), "output_sha256": sha256(out)}
        if whole:
            arrays[name] = out
        print(name, "done", flush=True)
    np.savez_compressed(OUT / "consec.npz", **arrays)
    (OUT / "consec.json").write_text(json.dumps(manifest, indent=1) + "\n")
    print("wrote", OUT / "consec.npz")


if __name__ == "__main__":
    main()
