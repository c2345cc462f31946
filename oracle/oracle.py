"""ctypes bindings of the CPU oracles (TEST INFRASTRUCTURE).

  Oracle     -> liboracle.so, the C restatement in tp_oracle.c
  Reference  -> _ref/libtpref.so, the reference library compiled from its own
                sources (oracle/Makefile); only present where it was built

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as a checker or a timed CPU baseline, never as the product path.
Also holds the seeded input generators shared by the tests, the golden-vector
script and the benchmark.
"""
from __future__ import annotations

import ctypes
import hashlib
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
P = 0xFFFFFFFF00000001
U64 = ctypes.c_uint64
U64P = ctypes.POINTER(ctypes.c_uint64)
VP = ctypes.c_void_p
CGGI_BINARY, CGGI_TERNARY, BMMP_BINARY = 0, 1, 2


def ptr(a: np.ndarray) -> U64P:
    assert a.dtype == np.uint64 and a.flags.c_contiguous
    return a.ctypes.data_as(U64P)


def sha256(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint64).tobytes()).hexdigest()


# ---------------------------------------------------------------------------
# seeded generators (splitmix64 streams, vectorised)
# ---------------------------------------------------------------------------
_G = np.uint64(0x9E3779B97F4A7C15)


def sm64(seed: int, count: int) -> np.ndarray:
    """count outputs of splitmix64 started at `seed` (the sampler's stream)."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed & (2**64 - 1)) + (np.arange(1, count + 1, dtype=np.uint64) * _G)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def uniform_mod(seed: int, count: int, q: int) -> np.ndarray:
    """Uniform residues mod q < 2^64 (the tiny modulo bias is irrelevant for test data)."""
    x = sm64(seed, count)
    if q == 0 or q == 2**64:
        return x
    if q & (q - 1) == 0:
        return x & np.uint64(q - 1)
    return np.array([int(v) % q for v in x], dtype=np.uint64) if count < 4096 else (
        (x >> np.uint64(1)) % np.uint64(q))


def lwe_secret(variant: int, n: int, N: int, seed: int) -> np.ndarray:
    """Binary key in {0,1}; ternary key in {0, 1, 2N-1} (-1 as in tests/cggi_blind_rotation_test.cpp:52)."""
    x = sm64(seed, n)
    if variant == CGGI_TERNARY:
        return np.array([0, 1, 2 * N - 1], dtype=np.uint64)[(x % np.uint64(3)).astype(np.int64)]
    return x & np.uint64(1)


def rlwe_secret(N: int, seed: int) -> np.ndarray:
    """Ternary RLWE key in {0, 1, p-1}."""
    x = sm64(seed, N)
    return np.array([0, 1, P - 1], dtype=np.uint64)[(x % np.uint64(3)).astype(np.int64)]


def lwe_inputs(N: int, n: int, count: int, seed: int) -> np.ndarray:
    """count x (n+1) LWE words uniform in [0, 2N)."""
    return (sm64(seed, count * (n + 1)) & np.uint64(2 * N - 1)).reshape(count, n + 1)


def lwe_encrypt_2n(key: np.ndarray, N: int, msgs, seed: int) -> np.ndarray:
    """Noise-free LWE mod 2N: b = <a, s> + m (mod 2N); key words taken mod 2N."""
    msgs = np.asarray(msgs, dtype=np.int64)
    n = key.size
    a = (sm64(seed, msgs.size * n) & np.uint64(2 * N - 1)).reshape(msgs.size, n).astype(np.int64)
    s = (key.astype(object) % (2 * N)).astype(np.int64)
    b = (a @ s + msgs) % (2 * N)
    return np.concatenate([a, b[:, None]], axis=1).astype(np.uint64)


def random_acc(N: int, count: int, seed: int) -> np.ndarray:
    """count x 2N uniformly random coefficient-domain RLWE words in [0, p)."""
    x = sm64(seed, count * 2 * N)
    x = np.where(x >= np.uint64(P), x - np.uint64(P), x)
    return x.reshape(count, 2 * N)


def lut_acc(N: int, table) -> np.ndarray:
    """Trivial RLWE (A = 0) of a test polynomial: table[k] repeated on N/len(table) coefficients."""
    table = np.asarray(table, dtype=object)
    per = N // len(table)
    B = np.array([int(table[i // per]) % P for i in range(N)], dtype=np.uint64)
    return np.concatenate([np.zeros(N, np.uint64), B])


# ---------------------------------------------------------------------------
# oracle (C restatement)
# ---------------------------------------------------------------------------
class Rng(ctypes.Structure):
    _fields_ = [("s", U64)]


def _build(target: str) -> None:
    subprocess.run(["make", "-s", "-C", str(HERE), target], check=True)


class Oracle:
    def __init__(self):
        so = HERE / "liboracle.so"
        if not so.exists() or so.stat().st_mtime < (HERE / "tp_oracle.c").stat().st_mtime:
            _build(str(so))
        L = ctypes.CDLL(str(so))
        D = ctypes.c_double
        I = ctypes.c_int
        R = ctypes.POINTER(Rng)
        sig = {
            "tpo_ntt_forward": (I, [U64, U64P, U64P]),
            "tpo_ntt_backward": (I, [U64, U64P, U64P]),
            "tpo_brk_words": (U64, [I, U64, U64, U64]),
            "tpo_br_keygen": (None, [R, I, U64, U64, U64, U64, D, U64P, U64P, U64P]),
            "tpo_br_keygen_aligned": (None, [R, I, U64, U64, U64, U64, D, U64P, U64P, U64P]),
            "tpo_blind_rotate": (I, [I, U64, U64, U64, U64, U64P, U64P, U64P, U64P, I]),
            "tpo_blind_rotate_many": (I, [I, U64, U64, U64, U64, U64P, U64P, U64P, U64P, U64, I, I]),
            "tpo_phase_rlwe": (None, [U64, U64P, U64P, U64P]),
            "tpo_signed_digits": (None, [U64P, U64P, U64, U64, U64]),
            "tpo_unsigned_digits": (None, [U64P, U64P, U64, U64, U64]),
            "tpo_make_rgsw": (None, [R, U64, D, U64P, U64P, U64P, U64, U64, I]),
            "tpo_make_rlwe": (None, [R, U64, D, U64P, U64P, U64P, I]),
            "tpo_rlwe_ks_keygen": (None, [R, U64, U64, U64, D, U64P, U64P, U64P]),
            "tpo_rlwe_ks": (None, [U64, U64, U64, U64P, U64P, U64P]),
            "tpo_lwe_ks_keygen": (None, [R, U64, U64, U64, U64, U64, D, U64P, U64P, U64P]),
            "tpo_lwe_ks": (None, [U64, U64, U64, U64, U64, U64P, U64P, U64P]),
            "tpo_make_lwe": (None, [R, U64, U64, D, U64P, U64, U64P]),
            "tpo_negacyclic_automorphism": (None, [U64P, U64P, U64, U64]),
            "tpo_auto_keygen": (None, [R, U64, U64, U64, D, U64, U64P, U64P]),
            "tpo_auto_eval": (None, [U64, U64, U64, U64, U64P, U64P, U64P]),
            "tpo_pack_keygen": (None, [R, U64, U64, U64, D, U64P, U64P]),
            "tpo_pack": (I, [U64, U64, U64, U64P, U64P, U64P, U64]),
            "tpo_sample_extract": (None, [U64P, U64P, U64, U64]),
            "tpo_pack_consecutive": (I, [U64, U64, U64, U64P, U64P, U64P, U64]),
            "tpo_trace_eval": (None, [U64, U64, U64, U64P, U64P, U64P]),
            "tpo_modulus_switch": (I, [U64P, U64, U64, U64, I]),
            "tpo_ss_test_poly": (I, [U64, U64, U64, U64P]),
            "tpo_ss_keygen": (None, [R, I, U64, U64, U64, U64, U64, U64, U64, U64, D, U64P, U64P, U64P, U64P,
                                     U64P]),
            "tpo_lwe_to_rgsw": (I, [I, U64, U64, U64, U64, U64P, U64, U64, U64P, U64, U64, U64P, U64, U64, U64P,
                                    U64P]),
            "tpo_ref_int_log2": (U64, [U64]),
            "tpo_sap_keygen": (None, [R, I, U64, U64, U64, U64, U64, U64, U64, U64, D, U64P, U64P, U64P, U64P,
                                      U64P]),
            "tpo_sap_homtrunc": (I, [U64, U64, U64, U64P, U64, U64P, U64P]),
            "tpo_sap_reset": (I, [I, U64, U64, U64, U64, U64P, U64, U64, U64P, U64, U64P]),
            "tpo_sap_decompose": (I, [I, U64, U64, U64, U64, U64P, U64, U64, U64P, U64, U64, U64P, U64, U64, U64,
                                      U64P, U64P, U64]),
            "tpo_psi": (U64, [U64]),
            "tpo_mul": (U64, [U64, U64]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        self.L = L

    # NTT
    def ntt_forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.uint64)
        out = np.empty_like(x)
        assert self.L.tpo_ntt_forward(x.size, ptr(out), ptr(x)) == 0
        return out

    def ntt_backward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.uint64)
        out = np.empty_like(x)
        assert self.L.tpo_ntt_backward(x.size, ptr(out), ptr(x)) == 0
        return out

    # blind rotation
    def br_keygen(self, variant, N, n, basis_log2, digits, std, lwe_key, rlwe_key, seed) -> np.ndarray:
        r = Rng(seed)
        brk = np.empty(self.L.tpo_brk_words(variant, N, n, digits), dtype=np.uint64)
        self.L.tpo_br_keygen(ctypes.byref(r), variant, N, n, basis_log2, digits, std,
                             ptr(np.ascontiguousarray(lwe_key, np.uint64)),
                             ptr(np.ascontiguousarray(rlwe_key, np.uint64)), ptr(brk))
        return brk

    def br_keygen_aligned(self, variant, N, n, basis_log2, digits, std, lwe_key, rlwe_key, seed) -> np.ndarray:
        """Key with RGSW rows scaled 2^(64 - beta(j+1)), aligned with the signed digits."""
        r = Rng(seed)
        brk = np.empty(self.L.tpo_brk_words(variant, N, n, digits), dtype=np.uint64)
        self.L.tpo_br_keygen_aligned(ctypes.byref(r), variant, N, n, basis_log2, digits, std,
                                     ptr(np.ascontiguousarray(lwe_key, np.uint64)),
                                     ptr(np.ascontiguousarray(rlwe_key, np.uint64)), ptr(brk))
        return brk

    def make_rlwe(self, N, std, msg, sk, seed) -> np.ndarray:
        """RLWE encryption (NTT domain) of a coefficient-domain message under sk (coefficients)."""
        r = Rng(seed)
        out = np.empty(2 * N, dtype=np.uint64)
        self.L.tpo_make_rlwe(ctypes.byref(r), N, std, ptr(out), ptr(np.ascontiguousarray(msg, np.uint64)),
                             ptr(self.ntt_forward(sk)), 0)
        return out

    def blind_rotate(self, variant, N, n, basis_log2, digits, brk, lwe, acc, out_coef) -> np.ndarray:
        res = np.empty(2 * N, dtype=np.uint64)
        rc = self.L.tpo_blind_rotate(variant, N, n, basis_log2, digits, ptr(brk),
                                     ptr(res), ptr(np.ascontiguousarray(lwe, np.uint64)),
                                     ptr(np.ascontiguousarray(acc, np.uint64)), int(out_coef))
        assert rc == 0
        return res

    def blind_rotate_many(self, variant, N, n, basis_log2, digits, brk, lwes, accs, out_coef, threads):
        lwes = np.ascontiguousarray(lwes, np.uint64)
        accs = np.ascontiguousarray(accs, np.uint64)
        res = np.empty((lwes.shape[0], 2 * N), dtype=np.uint64)
        rc = self.L.tpo_blind_rotate_many(variant, N, n, basis_log2, digits, ptr(brk), ptr(res), ptr(lwes),
                                          ptr(accs), lwes.shape[0], int(out_coef), threads)
        assert rc == 0
        return res

    # key switching
    def rlwe_ks_keygen(self, N, bl, dg, std, src, tgt, seed):
        r = Rng(seed)
        k = np.empty(dg * 2 * N, np.uint64)
        self.L.tpo_rlwe_ks_keygen(ctypes.byref(r), N, bl, dg, std, ptr(np.ascontiguousarray(src, np.uint64)),
                                  ptr(np.ascontiguousarray(tgt, np.uint64)), ptr(k))
        return k

    def rlwe_ks(self, N, bl, dg, ksk, inp, out=None):
        out = np.zeros(2 * N, np.uint64) if out is None else np.array(out, dtype=np.uint64)
        self.L.tpo_rlwe_ks(N, bl, dg, ptr(ksk), ptr(out), ptr(np.ascontiguousarray(inp, np.uint64)))
        return out

    def auto_keygen(self, N, bl, dg, std, index, key, seed):
        r = Rng(seed)
        k = np.empty(dg * 2 * N, np.uint64)
        self.L.tpo_auto_keygen(ctypes.byref(r), N, bl, dg, std, index, ptr(np.ascontiguousarray(key, np.uint64)),
                               ptr(k))
        return k

    def auto_eval(self, N, bl, dg, index, ksk, inp):
        out = np.zeros(2 * N, np.uint64)
        self.L.tpo_auto_eval(N, bl, dg, index, ptr(ksk), ptr(out), ptr(np.ascontiguousarray(inp, np.uint64)))
        return out

    def pack_keygen(self, N, bl, dg, std, key, seed):
        r = Rng(seed)
        logn = N.bit_length() - 1
        k = np.empty(logn * dg * 2 * N, np.uint64)
        self.L.tpo_pack_keygen(ctypes.byref(r), N, bl, dg, std, ptr(np.ascontiguousarray(key, np.uint64)), ptr(k))
        return k

    def pack(self, N, bl, dg, keys, lwes, length):
        out = np.empty(2 * N, np.uint64)
        assert self.L.tpo_pack(N, bl, dg, ptr(keys), ptr(out), ptr(np.ascontiguousarray(lwes, np.uint64)),
                               length) == 0
        return out

    def pack_consecutive(self, N, bl, dg, keys, lwes, length):
        out = np.empty(2 * N, np.uint64)
        assert self.L.tpo_pack_consecutive(N, bl, dg, ptr(keys), ptr(out),
                                           ptr(np.ascontiguousarray(lwes, np.uint64)), length) == 0
        return out

    def trace_eval(self, N, bl, dg, keys, rlwe_coef):
        """TraceEvaluator::Eval: NTT-domain result."""
        out = np.empty(2 * N, np.uint64)
        self.L.tpo_trace_eval(N, bl, dg, ptr(keys), ptr(out), ptr(np.ascontiguousarray(rlwe_coef, np.uint64)))
        return out

    def lwe_ks_keygen(self, q, n_in, n_out, bl, dg, std, src, tgt, seed):
        r = Rng(seed)
        k = np.empty(n_in * dg * (n_out + 1), np.uint64)
        self.L.tpo_lwe_ks_keygen(ctypes.byref(r), q, n_in, n_out, bl, dg, std,
                                 ptr(np.ascontiguousarray(src, np.uint64)), ptr(np.ascontiguousarray(tgt, np.uint64)),
                                 ptr(k))
        return k

    def lwe_ks(self, q, n_in, n_out, bl, dg, ksk, inp):
        out = np.zeros(n_out + 1, np.uint64)
        self.L.tpo_lwe_ks(q, n_in, n_out, bl, dg, ptr(ksk), ptr(out), ptr(np.ascontiguousarray(inp, np.uint64)))
        return out

    def modulus_switch(self, vec, source, target, kind) -> np.ndarray:
        """ModulusSwitch; kind 'round' | 'floor' | 'ceil'."""
        out = np.array(vec, dtype=np.uint64)
        assert self.L.tpo_modulus_switch(ptr(out), out.size, source, target,
                                         {"round": 0, "floor": 1, "ceil": 2}[kind]) == 0
        return out

    def sample_extract(self, rlwe: np.ndarray) -> np.ndarray:
        N = rlwe.size // 2
        out = np.zeros(N + 1, np.uint64)
        self.L.tpo_sample_extract(ptr(out), ptr(np.ascontiguousarray(rlwe, np.uint64)), 0, N)
        return out

    def pbs_epilogue(self, rlwe_coef, n_out, bl, dg, ksk, target):
        """SampleExtract (index 0) -> LWE key switch (fresh output) -> FLOOR switch to `target`."""
        N = rlwe_coef.size // 2
        ks = self.lwe_ks(P, N, n_out, bl, dg, ksk, self.sample_extract(rlwe_coef))
        return self.modulus_switch(ks, P, target, "floor")

    def ss_test_poly(self, N, out_digits, out_basis_log2) -> np.ndarray:
        """LWEtoRGSWConverter's m_acc = [0 | -tp | tp] (3N words)."""
        acc = np.empty(3 * N, np.uint64)
        assert self.L.tpo_ss_test_poly(N, out_digits, out_basis_log2, ptr(acc)) == 0
        return acc

    def ss_keygen(self, variant, N, n, br, tr, sq, std, lwe_key, rlwe_key, seed):
        """(rotation key, trace keys, squaring key) from one sampler stream, as the reference makes them."""
        r = Rng(seed)
        brk = np.empty(self.L.tpo_brk_words(variant, N, n, br[1]), np.uint64)
        logn = N.bit_length() - 1
        trk = np.empty(logn * tr[1] * 2 * N, np.uint64)
        sqk = np.empty(sq[1] * 2 * N, np.uint64)
        self.L.tpo_ss_keygen(ctypes.byref(r), variant, N, n, br[0], br[1], tr[0], tr[1], sq[0], sq[1], std,
                             ptr(np.ascontiguousarray(lwe_key, np.uint64)),
                             ptr(np.ascontiguousarray(rlwe_key, np.uint64)), ptr(brk), ptr(trk), ptr(sqk))
        return brk, trk, sqk

    def lwe_to_rgsw(self, variant, N, n, br, brk, tr, trace_keys, sq, sq_key, out_digits, out_basis_log2, lwe):
        """LWEtoRGSWConverter::Convert of one LWE; br/tr/sq = (basis_log2, digits) of each component."""
        out = np.empty(4 * N * out_digits, np.uint64)
        assert self.L.tpo_lwe_to_rgsw(variant, N, n, br[0], br[1], ptr(brk), tr[0], tr[1], ptr(trace_keys), sq[0],
                                      sq[1], ptr(sq_key), out_digits, out_basis_log2,
                                      ptr(np.ascontiguousarray(lwe, np.uint64)), ptr(out)) == 0
        return out

    def sap_keygen(self, variant, N, n, br, tr, ks, std, lwe_key, rlwe_key, seed):
        """(rotation key, trace keys, LWE key switch N -> n) from one sampler stream, as the reference makes them."""
        r = Rng(seed)
        brk = np.empty(self.L.tpo_brk_words(variant, N, n, br[1]), np.uint64)
        trk = np.empty((N.bit_length() - 1) * tr[1] * 2 * N, np.uint64)
        ksk = np.empty(N * ks[1] * (n + 1), np.uint64)
        self.L.tpo_sap_keygen(ctypes.byref(r), variant, N, n, br[0], br[1], tr[0], tr[1], ks[0], ks[1], std,
                              ptr(np.ascontiguousarray(lwe_key, np.uint64)),
                              ptr(np.ascontiguousarray(rlwe_key, np.uint64)), ptr(brk), ptr(trk), ptr(ksk))
        return brk, trk, ksk

    def sap_homtrunc(self, N, tr, trace_keys, radix, rlwe_ntt) -> np.ndarray:
        out = np.empty(2 * N, np.uint64)
        assert self.L.tpo_sap_homtrunc(N, tr[0], tr[1], ptr(trace_keys), radix, ptr(out),
                                       ptr(np.ascontiguousarray(rlwe_ntt, np.uint64))) == 0
        return out

    def sap_reset(self, variant, N, n, br, brk, ks, ksk, radix, acc_ntt) -> np.ndarray:
        acc = np.array(acc_ntt, dtype=np.uint64)
        assert self.L.tpo_sap_reset(variant, N, n, br[0], br[1], ptr(brk), ks[0], ks[1], ptr(ksk), radix,
                                    ptr(acc)) == 0
        return acc

    def sap_decompose(self, variant, N, n, br, brk, tr, trace_keys, ks, ksk, radix, beta, restart, lwe,
                      out_digits) -> np.ndarray:
        """SAPDecomposer::Decompose of one LWE: (digits, out_digits x (N+1) words, zero past the digits)."""
        out = np.zeros(out_digits * (N + 1), np.uint64)
        d = self.L.tpo_sap_decompose(variant, N, n, br[0], br[1], ptr(brk), tr[0], tr[1], ptr(trace_keys), ks[0],
                                     ks[1], ptr(ksk), radix, beta, restart,
                                     ptr(np.ascontiguousarray(lwe, np.uint64)), ptr(out), out_digits)
        assert d >= 0
        return d, out.reshape(out_digits, N + 1)

    def phase_rlwe(self, rlwe_ntt: np.ndarray, sk: np.ndarray) -> np.ndarray:
        N = sk.size
        sk_ntt = self.ntt_forward(sk)
        out = np.empty(N, dtype=np.uint64)
        self.L.tpo_phase_rlwe(N, ptr(out), ptr(np.ascontiguousarray(rlwe_ntt, np.uint64)), ptr(sk_ntt))
        return out


# ---------------------------------------------------------------------------
# reference library (compiled from the reference's own sources)
# ---------------------------------------------------------------------------
class Reference:
    PATH = HERE / "_ref" / "libtpref.so"

    @classmethod
    def available(cls) -> bool:
        return cls.PATH.exists()

    def __init__(self):
        if not self.PATH.exists():
            _build("ref")
        L = ctypes.CDLL(str(self.PATH))
        D = ctypes.c_double
        I = ctypes.c_int
        sig = {
            "ref_seed": (None, [U64]),
            "ref_ntt_forward": (I, [U64, U64P, U64P]),
            "ref_ntt_backward": (I, [U64, U64P, U64P]),
            "ref_br_create": (VP, [I, U64, U64, U64, U64, D, U64P, U64P]),
            "ref_br_key_words": (U64, [VP]),
            "ref_br_key_copy": (None, [VP, U64P]),
            "ref_br_rotate": (None, [VP, U64P, U64P, U64P, I]),
            "ref_br_rotate_many": (D, [VP, U64P, U64P, U64P, U64, I, I]),
            "ref_br_destroy": (None, [VP]),
            "ref_rlwe_ks_create": (VP, [U64, U64, U64, D, U64P, U64P]),
            "ref_rlwe_ks_key_copy": (None, [VP, U64P]),
            "ref_rlwe_ks_convert": (None, [VP, U64P, U64P]),
            "ref_rlwe_ks_destroy": (None, [VP]),
            "ref_lwe_ks_create": (VP, [U64, U64, U64, U64, U64, D, U64P, U64P]),
            "ref_lwe_ks_key_copy": (None, [VP, U64P]),
            "ref_lwe_ks_convert": (None, [VP, U64P, U64P]),
            "ref_lwe_ks_destroy": (None, [VP]),
            "ref_auto_create": (VP, [U64, U64, U64, D, ctypes.c_uint32, U64P]),
            "ref_auto_eval": (None, [VP, U64P, U64P]),
            "ref_auto_key_copy": (None, [VP, U64P]),
            "ref_auto_destroy": (None, [VP]),
            "ref_pack_create": (VP, [U64, U64, U64, D, U64P]),
            "ref_pack": (None, [VP, U64P, U64P, U64]),
            "ref_pack_key_copy": (None, [VP, U64P]),
            "ref_pack_consecutive": (None, [VP, U64P, U64P, U64]),
            "ref_trace_create": (VP, [U64, U64, U64, D, U64P]),
            "ref_trace_key_copy": (None, [VP, U64P]),
            "ref_trace_eval": (None, [VP, U64P, U64P]),
            "ref_trace_eval_auto": (None, [VP, U64P, U64P, U64]),
            "ref_trace_destroy": (None, [VP]),
            "ref_pack_destroy": (None, [VP]),
            "ref_sample_extract": (None, [U64P, U64P, U64, U64]),
            "ref_modulus_switch": (None, [U64P, U64, U64, U64, I]),
            "ref_ss_create": (VP, [I, U64, U64, U64, U64, U64, U64, U64, U64, D, U64, U64, U64P, U64P]),
            "ref_ss_key_words": (U64, [VP, I]),
            "ref_ss_key_copy": (None, [VP, I, U64P]),
            "ref_ss_convert": (None, [VP, U64P, U64P]),
            "ref_ss_test_poly": (None, [VP, U64P]),
            "ref_ss_destroy": (None, [VP]),
            "ref_sap_create": (VP, [I, U64, U64, U64, U64, U64, U64, U64, U64, D, U64, U64P, U64P]),
            "ref_sap_restart": (U64, [VP]),
            "ref_sap_set_restart": (None, [VP, U64]),
            "ref_sap_beta": (U64, [VP]),
            "ref_sap_key_words": (U64, [VP, I]),
            "ref_sap_key_copy": (None, [VP, I, U64P]),
            "ref_sap_decompose": (None, [VP, U64P, U64, U64P, U64]),
            "ref_sap_homtrunc": (None, [VP, U64P, U64P, U64]),
            "ref_sap_reset": (None, [VP, U64P, U64]),
            "ref_sap_destroy": (None, [VP]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        self.L = L
