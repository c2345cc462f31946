"""Golden blind rotations, key switches, automorphisms and packings at ring sizes above
4096, from the reference library itself.

Run here, where the reference sources exist: `python tests/golden/make_largen_golden.py
[br] [ks]` (default both; needs oracle/_ref/libtpref.so, see oracle/Makefile). The
reference's SolinasWorker accepts N up to 2^16; its rotators build a monomial table of
N (N + 2) words, so the rotation cases stop at N = 16384 (2.1 GB); the key-switching
cases go to 65536, the largest ring the worker accepts. Inputs and keys are
regenerated in the tests from the recorded seeds (same generators as make_golden.py);
outputs are recorded as SHA-256 of each result
(rotations: NTT-domain output, then coefficient output), with the key's SHA-256.
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
from oracle.oracle import (BMMP_BINARY, CGGI_BINARY, CGGI_TERNARY, P, Reference, lwe_secret, ptr,  # noqa: E402
                           random_acc, rlwe_secret, sha256, uniform_mod)

OUT = Path(__file__).resolve().parent

# (name, variant, N, n, basis_log2, digits, std)
CASES = [
    ("ternary_n8192", CGGI_TERNARY, 8192, 8, 12, 3, 3.2),
    ("binary_n8192_b16", CGGI_BINARY, 8192, 6, 16, 4, 3.2),
    ("bmmp_n8192", BMMP_BINARY, 8192, 6, 16, 4, 3.2),
    ("ternary_n16384", CGGI_TERNARY, 16384, 4, 12, 3, 3.2),
    ("binary_n16384_l2", CGGI_BINARY, 16384, 4, 20, 2, 3.2),
]

# (name, kind, N, basis_log2, digits, extra): extra = automorphism index or pack length
KS_CASES = [
    ("rks_n8192", "rlwe_ks", 8192, 16, 4, None),
    ("rks_n16384_b12", "rlwe_ks", 16384, 12, 3, None),
    ("rks_n32768", "rlwe_ks", 32768, 16, 4, None),
    ("auto5_n8192", "auto", 8192, 16, 4, 5),
    ("auto8193_n8192", "auto", 8192, 16, 4, 8193),
    ("auto3_n16384", "auto", 16384, 16, 4, 3),
    ("auto65535_n32768", "auto", 32768, 16, 4, 65535),
    ("pack16_n8192", "pack", 8192, 16, 4, 16),
    ("pack2_n16384", "pack", 16384, 16, 4, 2),
    ("pack4_n32768", "pack", 32768, 16, 4, 4),
    ("rks_n65536", "rlwe_ks", 65536, 16, 4, None),
    ("auto5_n65536", "auto", 65536, 16, 4, 5),
    ("pack2_n65536", "pack", 65536, 16, 4, 2),
]


def ks_section(L) -> dict:
    """Same key and input generators as make_golden.py's key-switching cases; the
    outputs of RLWEtoRLWEConverter::Convert (into zeroed outputs),
    AutomorphismEvaluator::Eval and LWEtoRLWEPacker::Pack, as SHA-256."""
    out = {}
    for name, kind, N, bl, dg, extra in KS_CASES:
        t0 = time.time()
        seed = case_seed(name)
        key = rlwe_secret(N, seed + 10)
        key2 = rlwe_secret(N, seed + 11)
        L.ref_seed(seed + 12)
        meta = {"kind": kind, "N": N, "basis_log2": bl, "digits": dg, "std": 3.2, "seed": seed, "key_seed": seed + 12}
        if kind in ("rlwe_ks", "auto"):
            if kind == "rlwe_ks":
                h = L.ref_rlwe_ks_create(N, bl, dg, 3.2, ptr(key), ptr(key2))
                copy, run, destroy = L.ref_rlwe_ks_key_copy, L.ref_rlwe_ks_convert, L.ref_rlwe_ks_destroy
            else:
                h = L.ref_auto_create(N, bl, dg, 3.2, extra, ptr(key))
                copy, run, destroy = L.ref_auto_key_copy, L.ref_auto_eval, L.ref_auto_destroy
                meta["index"] = extra
            ksk = np.empty(dg * 2 * N, np.uint64)
            copy(h, ptr(ksk))
            ins = random_acc(N, 2, seed + 1)
            sha = []
            for i in range(2):
                o = np.zeros(2 * N, np.uint64)
                run(h, ptr(o), ptr(np.ascontiguousarray(ins[i])))
                sha.append(sha256(o))
            destroy(h)
            meta.update(key_sha256=sha256(ksk), input_sha256=sha256(ins), out_sha256=sha)
        else:
            h = L.ref_pack_create(N, bl, dg, 3.2, ptr(key))
            logn = N.bit_length() - 1
            keys = np.empty(logn * dg * 2 * N, np.uint64)
            L.ref_pack_key_copy(h, ptr(keys))
            lwes = uniform_mod(seed + 1, extra * (N + 1), P).reshape(extra, N + 1)
            o = np.empty(2 * N, np.uint64)
            L.ref_pack(h, ptr(o), ptr(lwes), extra)
            L.ref_pack_destroy(h)
            meta.update(len=extra, key_sha256=sha256(keys), input_sha256=sha256(lwes), out_sha256=[sha256(o)])
        out[name] = meta
        print(f"{name}: {time.time() - t0:.1f}s", flush=True)
    return out


def main() -> None:
    L = Reference().L
    sections = set(sys.argv[1:]) or {"br", "ks"}
    path = OUT / "largen.json"
    manifest = json.loads(path.read_text()) if path.exists() else {}
    manifest.update({"generator": "tests/golden/make_largen_golden.py", "library": "oracle/_ref/libtpref.so"})
    if "ks" in sections:
        manifest["ks"] = ks_section(L)
    if "br" not in sections:
        path.write_text(json.dumps(manifest, indent=1) + "\n")
        return
    manifest["br"] = {}
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
    path.write_text(json.dumps(manifest, indent=1) + "\n")


if __name__ == "__main__":
    main()
