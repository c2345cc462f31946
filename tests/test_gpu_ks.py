"""Key switching, automorphisms, packing and LWE key switching on the GPU, bit-exact
against the reference's golden vectors and the C oracle."""
import json
from pathlib import Path

import numpy as np
import pytest

from kscases import ks_inputs, ks_key
from oracle.oracle import P, random_acc, rlwe_secret, sha256, sm64, uniform_mod

pytestmark = pytest.mark.gpu


def case(golden, name):
    return golden[0]["ks"][name], golden[1][f"ks_{name}"]


@pytest.mark.parametrize("tile", [4, 8])
@pytest.mark.parametrize("name", ["rlwe_ks_n2048", "rlwe_ks_n256_b12"])
def test_rlwe_ks_matches_reference(native, oracle, golden, name, tile):
    from fhetoothpaste_b200 import GpuRLWEtoRLWEConverter
    c, expect = case(golden, name)
    conv = GpuRLWEtoRLWEConverter(c["N"], 1 << c["basis_log2"], c["digits"], ks_key(oracle, name, c))
    conv.set_tile(tile)
    assert conv.tile == tile
    x = ks_inputs(c)
    out = np.zeros((2, 2 * c["N"]), np.uint64)
    conv.Convert(out, x)
    np.testing.assert_array_equal(out, expect)


def test_rlwe_ks_batch_accumulates_into_output(native, oracle, golden):
    """Convert subtracts into its output like the reference; a non-zero out is kept."""
    from fhetoothpaste_b200 import GpuRLWEtoRLWEConverter
    name = "rlwe_ks_n256_b12"
    c, _ = case(golden, name)
    N, k = c["N"], ks_key(oracle, name, c)
    conv = GpuRLWEtoRLWEConverter(N, 1 << c["basis_log2"], c["digits"], k)
    x = random_acc(N, 300, 31)
    base = random_acc(N, 300, 32)
    out = base.copy()
    conv.Convert(out, x)
    for b in (0, 150, 299):
        exp = oracle.rlwe_ks(N, c["basis_log2"], c["digits"], k, x[b], out=base[b])
        np.testing.assert_array_equal(out[b], exp)


@pytest.mark.parametrize("tile", [4, 8])
@pytest.mark.parametrize("name", ["auto5_n2048", "auto2049_n2048", "auto33_n128"])
def test_automorphism_matches_reference(native, oracle, golden, name, tile):
    from fhetoothpaste_b200 import GpuAutomorphismEvaluator
    c, expect = case(golden, name)
    ev = GpuAutomorphismEvaluator(c["N"], 1 << c["basis_log2"], c["digits"], c["index"], ks_key(oracle, name, c))
    ev.set_tile(tile)
    x = ks_inputs(c)
    out = np.zeros((2, 2 * c["N"]), np.uint64)
    ev.Eval(out, x)
    np.testing.assert_array_equal(out, expect)


@pytest.mark.parametrize("tile", [4, 8])
@pytest.mark.parametrize("name", ["pack2_n128", "pack32_n256", "pack2048_n2048"])
def test_pack_matches_reference(native, oracle, golden, name, tile):
    from fhetoothpaste_b200 import GpuLWEtoRLWEPacker
    c, expect = case(golden, name)
    pk = GpuLWEtoRLWEPacker(c["N"], 1 << c["basis_log2"], c["digits"], ks_key(oracle, name, c))
    pk.set_tile(tile)
    got = pk.Pack(ks_inputs(c), c["len"])
    np.testing.assert_array_equal(got[0], expect[0])


def test_pack_many_packs_against_oracle(native, oracle, golden):
    """Several packings in one batch (level-by-level over all packs), incl. trailing traces."""
    from fhetoothpaste_b200 import GpuLWEtoRLWEPacker
    name = "pack32_n256"
    c, _ = case(golden, name)
    N, k = c["N"], ks_key(oracle, name, c)
    pk = GpuLWEtoRLWEPacker(N, 1 << c["basis_log2"], c["digits"], k)
    for length in (2, 16, 256):
        packs = 3
        lwes = uniform_mod(50 + length, packs * length * (N + 1), P).reshape(packs * length, N + 1)
        got = pk.Pack(lwes, length)
        for p in range(packs):
            exp = oracle.pack(N, c["basis_log2"], c["digits"], k, lwes[p * length:(p + 1) * length], length)
            np.testing.assert_array_equal(got[p], exp, err_msg=f"len {length} pack {p}")


def test_packed_rlwe_decrypts_to_lwe_phases(native, oracle):
    """Packing invariant (tests/packing_tests.cpp:65-67): coefficient N/len * i of the
    packed RLWE's phase is the phase of input LWE i (noise-free keys, N/len scaling)."""
    from fhetoothpaste_b200 import GpuLWEtoRLWEPacker
    N, bl, dg, length = 256, 16, 4, 8
    s = rlwe_secret(N, 7)
    keys = oracle.pack_keygen(N, bl, dg, 0.0, s, 8)
    pk = GpuLWEtoRLWEPacker(N, 1 << bl, dg, keys)
    msgs = [(i * 1000003) % P for i in range(length)]
    lwes = np.zeros((length, N + 1), np.uint64)
    a = uniform_mod(9, length * N, P).reshape(length, N)
    for i in range(length):
        lwes[i, :N] = a[i]
        lwes[i, N] = (sum(int(x) * int(y) for x, y in zip(a[i], s)) + msgs[i]) % P
    packed = pk.Pack(lwes, length)[0]
    ntt = oracle.ntt_forward
    phase = oracle.phase_rlwe(np.concatenate([ntt(packed[:N]), ntt(packed[N:])]), s)
    for i in range(length):
        assert int(phase[i * (N // length)]) == msgs[i]


@pytest.mark.parametrize("name", ["lwe_ks_2048_630", "lwe_ks_64_16_b8"])
def test_lwe_ks_matches_reference(native, oracle, golden, name):
    from fhetoothpaste_b200 import GpuLWEtoLWEConverter
    c, expect = case(golden, name)
    conv = GpuLWEtoLWEConverter(c["n_in"], c["n_out"], 1 << c["basis_log2"], c["digits"], ks_key(oracle, name, c))
    x = ks_inputs(c)
    out = np.zeros((2, c["n_out"] + 1), np.uint64)
    conv.Convert(out, x)
    np.testing.assert_array_equal(out, expect)


def test_lwe_ks_large_batch_against_oracle(native, oracle, golden):
    from fhetoothpaste_b200 import GpuLWEtoLWEConverter
    name = "lwe_ks_64_16_b8"
    c, _ = case(golden, name)
    k = ks_key(oracle, name, c)
    conv = GpuLWEtoLWEConverter(c["n_in"], c["n_out"], 1 << c["basis_log2"], c["digits"], k)
    batch = 1000
    x = uniform_mod(77, batch * (c["n_in"] + 1), P).reshape(batch, c["n_in"] + 1)
    out = np.zeros((batch, c["n_out"] + 1), np.uint64)
    conv.Convert(out, x)
    for b in (0, 17, 999):
        np.testing.assert_array_equal(out[b], oracle.lwe_ks(P, c["n_in"], c["n_out"], c["basis_log2"], c["digits"],
                                                            k, x[b]))


CONSEC = json.loads((Path(__file__).resolve().parent / "golden" / "consec.json").read_text())


@pytest.mark.parametrize("name", sorted(CONSEC))
def test_pack_consecutive_matches_reference(native, oracle, name):
    """PackConsecutively (lwe_to_rlwe_packing.cpp:260-393) on the GPU against the reference's outputs,
    lengths 2 to N including non-powers of two; tile 8 on one case too."""
    from fhetoothpaste_b200 import GpuLWEtoRLWEPacker
    from test_consec_cpu import consec_case
    c = CONSEC[name]
    keys, lwes = consec_case(oracle, c)
    pk = GpuLWEtoRLWEPacker(c["N"], 1 << c["basis_log2"], c["digits"], keys)
    got = pk.PackConsecutively(lwes, c["len"])[0]
    assert sha256(got) == c["output_sha256"]
    if name == "consec100_n256":
        pk.set_tile(8)
        assert sha256(pk.PackConsecutively(lwes, c["len"])[0]) == c["output_sha256"]


def test_pack_consecutive_many_packs_and_decryption(native, oracle):
    """Several packings per call equal one-by-one oracle packings; with noise-free keys the packed
    phase holds message i at coefficient i and zeros after (packing_tests.cpp TestConsecutivePacking)."""
    from fhetoothpaste_b200 import GpuLWEtoRLWEPacker
    N, bl, dg, length, packs = 256, 16, 4, 24, 3
    z = (sm64(801, N) & np.uint64(1))
    keys = oracle.pack_keygen(N, bl, dg, 0.0, z, 802)
    rng = np.random.default_rng(803)
    lwes = np.zeros((packs * length, N + 1), np.uint64)
    zo = [int(v) for v in z]
    for r in range(packs * length):
        a = [int(v) for v in rng.integers(0, P, N, dtype=np.uint64)]
        lwes[r, :N] = a
        lwes[r, N] = (sum(x * s for x, s in zip(a, zo)) + (r % length) + 1000 * (r // length)) % P
    pk = GpuLWEtoRLWEPacker(N, 1 << bl, dg, keys)
    got = pk.PackConsecutively(lwes, length)
    for p in range(packs):
        want = oracle.pack_consecutive(N, bl, dg, keys, lwes[p * length:(p + 1) * length], length)
        np.testing.assert_array_equal(got[p], want, err_msg=f"pack {p}")
        phase = oracle.phase_rlwe(oracle_ntt_pair(oracle, got[p]), z)
        expect = np.zeros(N, np.uint64)
        expect[:length] = np.arange(length, dtype=np.uint64) + np.uint64(1000 * p)
        np.testing.assert_array_equal(phase, expect)


def oracle_ntt_pair(oracle, rlwe_coef):
    N = rlwe_coef.size // 2
    return np.concatenate([oracle.ntt_forward(rlwe_coef[:N]), oracle.ntt_forward(rlwe_coef[N:])])


TRACE = json.loads((Path(__file__).resolve().parent / "golden" / "trace.json").read_text())


@pytest.mark.parametrize("name", sorted(TRACE))
def test_trace_evaluator_matches_reference(native, oracle, name):
    """TraceEvaluator::Eval and EvalAuto (trace_evaluation.cpp:135-179) against the reference's outputs."""
    from fhetoothpaste_b200 import GpuTraceEvaluator
    from test_trace_cpu import trace_case
    c = TRACE[name]
    keys, x = trace_case(oracle, c)
    tr = GpuTraceEvaluator(c["N"], 1 << c["basis_log2"], c["digits"], keys)
    assert [sha256(r) for r in tr.Eval(x)] == c["eval_sha256"]
    for t, want in zip(c["auto_index"], c["auto_sha256"]):
        assert sha256(tr.EvalAuto(x[:1], t)[0]) == want, f"index {t}"
