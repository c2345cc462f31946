"""Blind rotation at ring sizes above 4096 on the GPU: one rotation per cluster of 2, 4, 8 or 16
CTAs with the transforms distributed over distributed shared memory (csrc/cluster_ntt.cuh).
Bit-exact against the reference library's outputs (tests/golden/largen.json, N = 8192 and
16384: SHA-256 of every output word) and against the C oracle (pinned to those outputs by
tests/test_largen_oracle_cpu.py) at N = 32768 and 65536 and on batches larger than the resident
grid; key switching, automorphisms, packing and transforms up to N = 65536."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import BMMP_BINARY, CGGI_BINARY, CGGI_TERNARY, lwe_inputs, lwe_secret, random_acc, rlwe_secret, \
    sha256

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden" / "largen.json"
CASES = json.loads(GOLDEN.read_text())["br"]


def _rotator(oracle, v, N, n, bl, dg, seed):
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    brk = oracle.br_keygen(v, N, n, bl, dg, 3.2, lwe_secret(v, n, N, seed), rlwe_secret(N, seed + 1), seed + 2)
    return brk, GpuBlindRotator(BlindRotationContext(v, N, n, 1 << bl, dg), brk)


@pytest.mark.parametrize("name", sorted(CASES))
def test_large_ring_matches_reference(native, oracle, name):
    import sys
    sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
    from make_golden import br_inputs
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    c = CASES[name]
    N, n, v = c["N"], c["n"], c["variant"]
    lk, rk = lwe_secret(v, n, N, c["seed"] + 10), rlwe_secret(N, c["seed"] + 11)
    brk = oracle.br_keygen(v, N, n, c["basis_log2"], c["digits"], c["std"], lk, rk, c["key_seed"])
    rot = GpuBlindRotator(BlindRotationContext(v, N, n, 1 << c["basis_log2"], c["digits"]), brk)
    lwes, accs, coefs = br_inputs(name, N, n, c["seed"])
    assert rot.mac_form == 0  # row-by-row is the default on a cluster
    for form in (0, 1):
        if form == 1:
            try:
                rot.set_mac_form(1)   # the digit-staged form, where it fits
            except Exception:
                continue
        else:
            rot.set_mac_form(0)
        for i, oc in enumerate(coefs):
            res = np.zeros(2 * N, np.uint64)
            rot.BlindRotate(res, np.ascontiguousarray(lwes[i]), np.ascontiguousarray(accs[i]), bool(oc))
            assert sha256(res) == c["out_sha256"][i], (name, form, i)
    rot.close()


@pytest.mark.parametrize("N", [32768, 65536])
@pytest.mark.parametrize("v,bl,dg", [(CGGI_TERNARY, 12, 3), (CGGI_BINARY, 16, 4), (BMMP_BINARY, 16, 4)])
def test_largest_rings_match_oracle(native, oracle, v, bl, dg, N):
    """N = 32768 (8 CTAs of 4096 coefficients) and 65536 (16 CTAs of 4096), where the
    reference's rotators cannot build their N (N + 2)-word monomial table: the oracle,
    pinned to the reference at 8192 and 16384."""
    n = 4 if N == 32768 else 2
    brk, rot = _rotator(oracle, v, N, n, bl, dg, 500 + v)
    lwes = lwe_inputs(N, n, 2, 510)
    accs = random_acc(N, 2, 511)
    for oc in (0, 1):
        got = rot.blind_rotate_batch_host(lwes, accs, out_coef=bool(oc))
        for b in range(2):
            want = oracle.blind_rotate(v, N, n, bl, dg, brk, lwes[b], accs[b], oc)
            np.testing.assert_array_equal(got[b], want, err_msg=f"out_coef {oc}, ciphertext {b}")
    rot.close()


def test_cluster_batch_larger_than_the_grid(native, oracle):
    """More rotations than resident clusters: clusters loop over the batch."""
    N, n, bl, dg = 8192, 6, 12, 3
    brk, rot = _rotator(oracle, CGGI_TERNARY, N, n, bl, dg, 520)
    batch = 2 * (148 // 4) + 5
    lwes = lwe_inputs(N, n, batch, 521)
    accs = random_acc(N, batch, 522)
    got = rot.blind_rotate_batch_host(lwes, accs)
    for b in (0, 1, 36, 37, batch - 1):
        np.testing.assert_array_equal(got[b], oracle.blind_rotate(CGGI_TERNARY, N, n, bl, dg, brk, lwes[b],
                                                                   accs[b], 0), err_msg=f"ciphertext {b}")
    rot.close()


def test_cluster_sizes_refuse_other_tiles(native, oracle):
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator, _native
    N, n = 16384, 2
    brk = np.zeros(BlindRotationContext(CGGI_BINARY, N, n, 1 << 16, 4).key_words(), np.uint64)
    rot = GpuBlindRotator(BlindRotationContext(CGGI_BINARY, N, n, 1 << 16, 4), brk)
    assert rot.tile == 4 and rot.split == 1
    with pytest.raises(_native.TpError):
        rot.set_tile(8)
    with pytest.raises(_native.TpError):
        rot.set_split(2)
    rot.close()


KS_CASES = json.loads(GOLDEN.read_text())["ks"]


@pytest.mark.parametrize("name", sorted(KS_CASES))
def test_large_ring_key_switching_matches_reference(native, oracle, name):
    """RLWEtoRLWEConverter::Convert, AutomorphismEvaluator::Eval and LWEtoRLWEPacker::Pack at
    N = 8192 .. 65536 (one item per cluster of 2, 4, 8 or 16 CTAs) against the reference's outputs."""
    from kscases import ks_inputs, ks_key
    from fhetoothpaste_b200 import GpuAutomorphismEvaluator, GpuLWEtoRLWEPacker, GpuRLWEtoRLWEConverter
    c = KS_CASES[name]
    N, base, dg = c["N"], 1 << c["basis_log2"], c["digits"]
    key, x = ks_key(oracle, name, c), ks_inputs(c)
    if c["kind"] == "pack":
        op = GpuLWEtoRLWEPacker(N, base, dg, key)
        got = [op.Pack(x, c["len"])[0]]
    else:
        op = (GpuRLWEtoRLWEConverter(N, base, dg, key) if c["kind"] == "rlwe_ks"
              else GpuAutomorphismEvaluator(N, base, dg, c["index"], key))
        assert op.tile == 4
        out = np.zeros((2, 2 * N), np.uint64)
        (op.Convert if c["kind"] == "rlwe_ks" else op.Eval)(out, x)
        got = list(out)
    assert [sha256(np.ascontiguousarray(g)) for g in got] == c["out_sha256"], name
    op.close()


def test_large_ring_key_switch_batch_larger_than_the_grid(native, oracle):
    """More key switches than resident clusters, accumulated into a non-zero output."""
    from kscases import ks_key
    from fhetoothpaste_b200 import GpuRLWEtoRLWEConverter
    name = "rks_n8192"
    c = KS_CASES[name]
    N, bl, dg = c["N"], c["basis_log2"], c["digits"]
    k = ks_key(oracle, name, c)
    conv = GpuRLWEtoRLWEConverter(N, 1 << bl, dg, k)
    with pytest.raises(Exception):
        conv.set_tile(8)
    batch = 3 * (148 // 4) + 7
    x = random_acc(N, batch, 530)
    base = random_acc(N, batch, 531)
    out = base.copy()
    conv.Convert(out, x)
    for b in (0, 36, 37, 111, batch - 1):
        np.testing.assert_array_equal(out[b], oracle.rlwe_ks(N, bl, dg, k, x[b], out=base[b]), err_msg=f"item {b}")
    conv.close()


@pytest.mark.parametrize("N", [8192, 16384, 32768, 65536])
def test_large_ring_ntt_matches_oracle(native, oracle, N):
    """The standalone transforms on a cluster: forward against the oracle, backward inverts it
    (out of place and in place, several polynomials)."""
    import torch
    from fhetoothpaste_b200 import ntt_backward, ntt_forward
    count = 5
    x = random_acc(N // 2, count, 540 + N)  # count x N words below p
    d_in = torch.from_numpy(x.view(np.int64)).cuda()
    d_out = torch.empty_like(d_in)
    ntt_forward(N, count, d_out.data_ptr(), d_in.data_ptr())
    got = d_out.cpu().numpy().view(np.uint64)
    for b in (0, count - 1):
        np.testing.assert_array_equal(got[b], oracle.ntt_forward(x[b]), err_msg=f"forward {b}")
    ntt_backward(N, count, d_out.data_ptr(), d_out.data_ptr())
    np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint64), x)


def test_large_ring_trace_and_consecutive_packing_match_oracle(native, oracle):
    """TraceEvaluator::Eval and PackConsecutively (a non-power-of-two length) at N = 8192."""
    from fhetoothpaste_b200 import GpuLWEtoRLWEPacker, GpuTraceEvaluator
    from oracle.oracle import P, uniform_mod
    N, bl, dg = 8192, 16, 4
    keys = oracle.pack_keygen(N, bl, dg, 3.2, rlwe_secret(N, 550), 551)
    x = random_acc(N, 2, 552)
    tr = GpuTraceEvaluator(N, 1 << bl, dg, keys)
    got = tr.Eval(x)
    for b in range(2):
        np.testing.assert_array_equal(got[b], oracle.trace_eval(N, bl, dg, keys, x[b]), err_msg=f"trace {b}")
    tr.close()
    length = 11
    lwes = uniform_mod(553, length * (N + 1), P).reshape(length, N + 1)
    pk = GpuLWEtoRLWEPacker(N, 1 << bl, dg, keys)
    np.testing.assert_array_equal(pk.PackConsecutively(lwes, length)[0],
                                  oracle.pack_consecutive(N, bl, dg, keys, lwes, length))
    pk.close()


def test_large_ring_scheme_switching_and_sap_match_oracle(native, oracle, cuda):
    """The composite operators on the cluster kernels at N = 8192: LWEtoRGSWConverter::Convert
    (rotation, trace, squaring key switch) and SAPDecomposer::Decompose (rotations, truncation
    tree, LWE key switch), against the oracle restatement."""
    from fhetoothpaste_b200 import GpuLWEtoRGSWConverter, GpuSAPDecomposer
    N, n = 8192, 4
    sk = lwe_secret(CGGI_BINARY, n, N, 560)
    z = rlwe_secret(N, 561)
    g = (16, 4)
    keys = oracle.ss_keygen(CGGI_BINARY, N, n, g, g, g, 3.2, sk, z, 562)
    conv = GpuLWEtoRGSWConverter((CGGI_BINARY, N, n, 1 << 16, 4), (1 << 16, 4), (1 << 16, 4), 4, 1 << 16, *keys)
    lwes = lwe_inputs(N, n, 2, 563)
    got = conv.Convert(lwes)
    for j in range(2):
        want = oracle.lwe_to_rgsw(CGGI_BINARY, N, n, g, keys[0], g, keys[1], g, keys[2], 4, 16, lwes[j])
        np.testing.assert_array_equal(got[j], want, err_msg=f"LWE->RGSW input {j}")
    skeys = oracle.sap_keygen(CGGI_BINARY, N, n, g, g, g, 3.2, sk, z, 564)
    beta = int(np.count_nonzero(sk))
    dec = GpuSAPDecomposer((CGGI_BINARY, N, n, 1 << 16, 4), (1 << 16, 4), (1 << 16, 4), *skeys,
                           hamming_weight=beta, restart_period=4)
    small = np.random.default_rng(565).integers(0, 1 << 12, (2, n + 1), dtype=np.uint64)
    digits, outs = dec.Decompose(small, 16, 4)
    for j in range(1):  # the oracle takes about 17 s per input at this size
        d, want = oracle.sap_decompose(CGGI_BINARY, N, n, g, skeys[0], g, skeys[1], g, skeys[2], 16, beta, 4,
                                       small[j], 4)
        assert digits[j] == d
        np.testing.assert_array_equal(outs[j], want, err_msg=f"SAP input {j}")
