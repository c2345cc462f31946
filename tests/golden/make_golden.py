"""Generates the golden vectors in tests/golden/ from the reference library itself.

Run here, where the reference sources exist: `python tests/golden/make_golden.py`.
It builds oracle/_ref/libtpref.so (the reference compiled from its own sources
with the sampler/HEXL shims, see oracle/Makefile), feeds it seeded inputs and
records its outputs. Inputs are not stored: tests regenerate them from the
recorded seeds with oracle/oracle.py's generators and check the recorded input
hashes. Keys are regenerated by the C oracle from the same sampler seed and must
hash to the reference key's recorded SHA-256.
"""
from __future__ import annotations

import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle.oracle import (BMMP_BINARY, CGGI_BINARY, CGGI_TERNARY, P, Reference, lwe_encrypt_2n,  # noqa: E402
                           lwe_inputs, lwe_secret, ptr, random_acc, rlwe_secret, sha256, sm64, uniform_mod)

OUT = Path(__file__).resolve().parent

# (name, variant, N, n, basis_log2, digits, std)
BR_CASES = [
    ("small_binary_n256", CGGI_BINARY, 256, 16, 12, 3, 3.2),
    ("small_ternary_n128", CGGI_TERNARY, 128, 10, 16, 4, 3.2),
    ("small_bmmp_n512", BMMP_BINARY, 512, 12, 16, 3, 3.2),
    ("cfg1_binary_n1024", CGGI_BINARY, 1024, 500, 16, 4, 3.2),
    ("cfg2_ternary_n2048", CGGI_TERNARY, 2048, 630, 12, 3, 3.2),
    ("cfg3_bmmp_n2048", BMMP_BINARY, 2048, 768, 16, 4, 3.2),
    ("cfg5a_ternary_n1024", CGGI_TERNARY, 1024, 500, 12, 3, 3.2),
    ("cfg5c_ternary_n4096", CGGI_TERNARY, 4096, 900, 12, 3, 3.2),
]


# (name, kind, N, basis_log2, digits, extra): extra = automorphism index, pack length or (n_in, n_out)
KS_CASES = [
    ("rlwe_ks_n2048", "rlwe_ks", 2048, 16, 4, None),
    ("rlwe_ks_n256_b12", "rlwe_ks", 256, 12, 3, None),
    ("auto5_n2048", "auto", 2048, 16, 4, 5),
    ("auto2049_n2048", "auto", 2048, 16, 4, 2049),
    ("auto33_n128", "auto", 128, 16, 4, 33),
    ("pack2_n128", "pack", 128, 16, 4, 2),
    ("pack32_n256", "pack", 256, 16, 4, 32),
    ("pack2048_n2048", "pack", 2048, 16, 4, 2048),
    ("lwe_ks_2048_630", "lwe_ks", 0, 16, 4, (2048, 630)),
    ("lwe_ks_64_16_b8", "lwe_ks", 0, 8, 3, (64, 16)),
]


def br_inputs(name: str, N: int, n: int, seed: int):
    """Two rotations per case: edge-valued LWE words with a random acc (NTT-domain
    output), then uniform words with another random acc (coefficient output)."""
    lwes = lwe_inputs(N, n, 2, seed + 1)
    lwes[0, 0] = 0
    lwes[0, 1 % n] = N
    lwes[0, 2 % n] = 2 * N - 1
    lwes[0, n] = N + 5
    accs = random_acc(N, 2, seed + 2)
    return lwes, accs, [0, 1]


def lwe_ks_secrets(n_in: int, n_out: int, seed: int):
    """Ternary LWE secrets mod p (-1 as p-1) for the LWE key-switching cases."""
    def tern(n, sd):
        x = sm64(sd, n) % np.uint64(3)
        return np.array([0, 1, P - 1], dtype=np.uint64)[x.astype(np.int64)]
    return tern(n_in, seed + 10), tern(n_out, seed + 11)


def case_seed(name: str) -> int:
    return int.from_bytes(name.encode()[:8].ljust(8, b"\0"), "little") & 0x7FFFFFFFFFFFFFFF


def main() -> None:
    ref = Reference()
    L = ref.L
    manifest = {"generator": "tests/golden/make_golden.py", "library": "oracle/_ref/libtpref.so",
                "ntt": {}, "br": {}}
    arrays = {}

    # NTT
    for logn in range(7, 13):
        N = 1 << logn
        x = uniform_mod(1000 + logn, N, P)
        f = np.empty(N, np.uint64)
        b = np.empty(N, np.uint64)
        assert L.ref_ntt_forward(N, ptr(f), ptr(x)) == 0
        assert L.ref_ntt_backward(N, ptr(b), ptr(x)) == 0
        arrays[f"ntt_fwd_{N}"] = f
        arrays[f"ntt_bwd_{N}"] = b
        manifest["ntt"][str(N)] = {"seed": 1000 + logn, "input_sha256": sha256(x)}

    # Blind rotation
    for name, variant, N, n, bl, dg, std in BR_CASES:
        t0 = time.time()
        seed = case_seed(name)
        lk = lwe_secret(variant, n, N, seed + 10)
        rk = rlwe_secret(N, seed + 11)
        key_seed = seed + 12
        L.ref_seed(key_seed)
        h = L.ref_br_create(variant, N, n, bl, dg, std, ptr(lk), ptr(rk))
        kw = L.ref_br_key_words(h)
        brk = np.empty(kw, np.uint64)
        L.ref_br_key_copy(h, ptr(brk))
        lwes, accs, coefs = br_inputs(name, N, n, seed)
        results = []
        for i, oc in enumerate(coefs):
            r = np.empty(2 * N, np.uint64)
            L.ref_br_rotate(h, ptr(r), ptr(np.ascontiguousarray(lwes[i])), ptr(np.ascontiguousarray(accs[i])), oc)
            results.append(r)
        L.ref_br_destroy(h)
        arrays[f"br_{name}"] = np.stack(results)
        manifest["br"][name] = {
            "variant": variant, "N": N, "n": n, "basis_log2": bl, "digits": dg, "std": std, "seed": seed,
            "key_seed": key_seed, "key_words": int(kw), "key_sha256": sha256(brk),
            "lwe_sha256": sha256(lwes), "acc_sha256": sha256(accs), "out_coef": coefs,
        }
        print(f"{name}: {time.time() - t0:.1f}s", flush=True)

    # Key switching, automorphisms, packing, LWE key switching
    manifest["ks"] = {}
    for name, kind, N, bl, dg, extra in KS_CASES:
        t0 = time.time()
        seed = case_seed(name)
        key = rlwe_secret(N, seed + 10)
        key2 = rlwe_secret(N, seed + 11)
        L.ref_seed(seed + 12)
        meta = {"kind": kind, "N": N, "basis_log2": bl, "digits": dg, "std": 3.2, "seed": seed, "key_seed": seed + 12}
        if kind == "rlwe_ks":
            h = L.ref_rlwe_ks_create(N, bl, dg, 3.2, ptr(key), ptr(key2))
            ksk = np.empty(dg * 2 * N, np.uint64)
            L.ref_rlwe_ks_key_copy(h, ptr(ksk))
            ins = random_acc(N, 2, seed + 1)
            outs = []
            for i in range(2):
                o = np.zeros(2 * N, np.uint64)
                L.ref_rlwe_ks_convert(h, ptr(o), ptr(np.ascontiguousarray(ins[i])))
                outs.append(o)
            L.ref_rlwe_ks_destroy(h)
            meta.update(key_sha256=sha256(ksk), input_sha256=sha256(ins))
        elif kind == "auto":
            h = L.ref_auto_create(N, bl, dg, 3.2, extra, ptr(key))
            ksk = np.empty(dg * 2 * N, np.uint64)
            L.ref_auto_key_copy(h, ptr(ksk))
            ins = random_acc(N, 2, seed + 1)
            outs = []
            for i in range(2):
                o = np.zeros(2 * N, np.uint64)
                L.ref_auto_eval(h, ptr(o), ptr(np.ascontiguousarray(ins[i])))
                outs.append(o)
            L.ref_auto_destroy(h)
            meta.update(index=extra, key_sha256=sha256(ksk), input_sha256=sha256(ins))
        elif kind == "pack":
            h = L.ref_pack_create(N, bl, dg, 3.2, ptr(key))
            logn = N.bit_length() - 1
            keys = np.empty(logn * dg * 2 * N, np.uint64)
            L.ref_pack_key_copy(h, ptr(keys))
            length = extra
            lwes = uniform_mod(seed + 1, length * (N + 1), P).reshape(length, N + 1)
            o = np.empty(2 * N, np.uint64)
            L.ref_pack(h, ptr(o), ptr(lwes), length)
            outs = [o]
            L.ref_pack_destroy(h)
            meta.update(len=length, key_sha256=sha256(keys), input_sha256=sha256(lwes))
        else:  # lwe_ks: extra = (n_in, n_out)
            n_in, n_out = extra
            src, tgt = lwe_ks_secrets(n_in, n_out, seed)
            ins = uniform_mod(seed + 1, 2 * (n_in + 1), P).reshape(2, n_in + 1)
            outs = []
            # One fresh converter per input: LWEtoLWEConverter::Convert clears only
            # the first (n_out + 8) / 8 accumulator words between calls
            # (ZERO_UINT64_ARR(m_acc.data(), n_out + 1) at lwe_conversion.cpp:217
            # expands to memset(.., n_out + 1 * sizeof(uint64_t))), so only a
            # converter's first call gives the intended result.
            for i in range(2):
                L.ref_seed(seed + 12)
                h = L.ref_lwe_ks_create(P, n_in, n_out, bl, dg, 3.2, ptr(src), ptr(tgt))
                ksk = np.empty(n_in * dg * (n_out + 1), np.uint64)
                L.ref_lwe_ks_key_copy(h, ptr(ksk))
                o = np.zeros(n_out + 1, np.uint64)
                L.ref_lwe_ks_convert(h, ptr(o), ptr(np.ascontiguousarray(ins[i])))
                outs.append(o)
                L.ref_lwe_ks_destroy(h)
            meta.update(n_in=n_in, n_out=n_out, key_sha256=sha256(ksk), input_sha256=sha256(ins))
        arrays[f"ks_{name}"] = np.stack(outs)
        manifest["ks"][name] = meta
        print(f"{name}: {time.time() - t0:.1f}s", flush=True)

    np.savez(OUT / "golden.npz", **arrays)
    (OUT / "golden.json").write_text(json.dumps(manifest, indent=1) + "\n")
    print("wrote", OUT / "golden.npz", OUT / "golden.json")


if __name__ == "__main__":
    main()
