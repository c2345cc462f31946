"""Blind rotation at ring sizes above 4096 on the GPU: one rotation per cluster of 4, 8 or 16
CTAs with the transforms distributed over distributed shared memory (csrc/cluster_ntt.cuh).
Bit-exact against the reference library's outputs (tests/golden/largen.json, N = 8192 and
16384: SHA-256 of every output word) and against the C oracle (pinned to those outputs by
tests/test_largen_oracle_cpu.py) at N = 32768 and on batches larger than the resident grid."""
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


@pytest.mark.parametrize("v,bl,dg", [(CGGI_TERNARY, 12, 3), (CGGI_BINARY, 16, 4), (BMMP_BINARY, 16, 4)])
def test_n32768_matches_oracle(native, oracle, v, bl, dg):
    N, n = 32768, 4
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
