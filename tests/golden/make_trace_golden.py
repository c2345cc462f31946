"""Golden vectors for TraceEvaluator::Eval / EvalAuto (lib/src/operators/trace_evaluation.cpp:
135-179) from the reference library built in oracle/_ref. Run in the container that has the
reference build:

    python tests/golden/make_trace_golden.py

Keys come from the shimmed sampler seeded with `key_seed` (SHA-256 recorded; the oracle's
packing key generation makes the same keys); inputs are uniform coefficient-domain RLWEs
regenerated from `in_seed`. EvalAuto is recorded for the pointer overload.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle.oracle import Reference, ptr, random_acc, rlwe_secret, sha256  # noqa: E402

OUT = Path(__file__).resolve().parent

# name, N, basis_log2, digits, automorphism indices for EvalAuto
CASES = [
    ("trace_n256", 256, 16, 4, [3, 17, 257]),
    ("trace_n128_b12", 128, 12, 3, [5, 129]),
    ("trace_n2048", 2048, 16, 4, [3, 2049]),
]


def main() -> None:
    L = Reference().L
    manifest, arrays = {}, {}
    for i, (name, N, bl, dg, idx) in enumerate(CASES):
        key_seed, in_seed, sk_seed = 500 + i, 530 + i, 560 + i
        key = rlwe_secret(N, sk_seed)
        L.ref_seed(key_seed)
        h = L.ref_trace_create(N, bl, dg, 3.2, ptr(key))
        keys = np.empty((N.bit_length() - 1) * dg * 2 * N, np.uint64)
        L.ref_trace_key_copy(h, ptr(keys))
        x = random_acc(N, 2, in_seed)
        outs = np.empty((2, 2 * N), np.uint64)
        for j in range(2):
            L.ref_trace_eval(h, ptr(outs[j]), ptr(np.ascontiguousarray(x[j])))
        autos = np.zeros((len(idx), 2 * N), np.uint64)
        for j, t in enumerate(idx):
            L.ref_trace_eval_auto(h, ptr(autos[j]), ptr(np.ascontiguousarray(x[0])), t)
        L.ref_trace_destroy(h)
        manifest[name] = {"N": N, "basis_log2": bl, "digits": dg, "std": 3.2, "key_seed": key_seed,
                          "in_seed": in_seed, "sk_seed": sk_seed, "auto_index": idx, "key_sha256": sha256(keys),
                          "input_sha256": sha256(x), "eval_sha256": [sha256(o) for o in outs],
                          "auto_sha256": [sha256(a) for a in autos]}
        if N <= 256:
            arrays[name] = outs
        print(name, "done", flush=True)
    np.savez_compressed(OUT / "trace.npz", **arrays)
    (OUT / "trace.json").write_text(json.dumps(manifest, indent=1) + "\n")
    print("wrote", OUT / "trace.npz")


if __name__ == "__main__":
    main()
