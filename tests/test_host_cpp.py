"""The C++ drop-in operators (fhetoothpaste_b200/host): key generation equals the
oracle's for the same seed (CPU), the reference's parameter checks throw (CPU), and
rotations / packing through the C++ classes equal the oracle (GPU)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import (CGGI_BINARY, CGGI_TERNARY, BMMP_BINARY, lwe_inputs, lwe_secret, random_acc,
                           rlwe_secret, sm64)

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "fhetoothpaste_b200"


@pytest.fixture(scope="session")
def driver(tmp_path_factory):
    from fhetoothpaste_b200 import build
    build.build_gpu()
    build.build_host()
    exe = tmp_path_factory.mktemp("cpp") / "host_ops_driver"
    subprocess.run(["g++", "-std=c++20", "-O2", f"-I{ROOT / 'include'}", f"-I{PKG / 'host'}",
                    str(ROOT / "tests" / "cpp" / "host_ops_driver.cpp"), "-o", str(exe), f"-L{PKG}",
                    "-ltoothpaste_host", "-ltoothpaste_gpu", f"-Wl,-rpath,{PKG}"], check=True)
    return exe


def run(exe, tmp, *args):
    """Runs the driver; array arguments are written to files and the last one is read back."""
    argv = [str(exe)]
    for i, a in enumerate(args):
        if isinstance(a, np.ndarray):
            f = tmp / f"in{i}.bin"
            np.ascontiguousarray(a, np.uint64).tofile(f)
            argv.append(str(f))
        else:
            argv.append(str(a))
    out = tmp / "out.bin"
    argv.append(str(out))
    res = subprocess.run(argv, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return np.fromfile(out, dtype=np.uint64)


BR_SMALL = [  # (variant, N, n, beta, digits, std)
    (CGGI_BINARY, 256, 12, 16, 3, 3.2),
    (CGGI_TERNARY, 128, 10, 20, 2, 3.2),
    (BMMP_BINARY, 256, 12, 12, 4, 3.2),
]


@pytest.mark.parametrize("case", BR_SMALL, ids=["binary", "ternary", "bmmp"])
def test_keygen_equals_oracle(driver, oracle, tmp_path, case):
    variant, N, n, beta, digits, std = case
    sk = lwe_secret(variant, n, N, seed=41)
    z = rlwe_secret(N, seed=42)
    got = run(driver, tmp_path, "keygen-br", variant, N, n, beta, digits, std, 7, sk, z)
    want = oracle.br_keygen(variant, N, n, beta, digits, std, sk, z, seed=7)
    assert got.size == want.size
    assert np.array_equal(got, want)


def test_packing_keygen_equals_oracle(driver, oracle, tmp_path):
    N, beta, digits, std = 128, 16, 4, 3.2
    z = rlwe_secret(N, seed=9)
    got = run(driver, tmp_path, "keygen-pack", N, beta, digits, std, 11, z)
    want = oracle.pack_keygen(N, beta, digits, std, z, seed=11)
    assert np.array_equal(got, want)


def test_parameter_checks_throw(driver):
    res = subprocess.run([str(driver), "errors"], capture_output=True, text=True)
    assert res.returncode == 0 and res.stdout.startswith("ok"), res.stdout + res.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("case", BR_SMALL, ids=["binary", "ternary", "bmmp"])
def test_cpp_operator_rotates_like_oracle(driver, oracle, cuda, tmp_path, case):
    variant, N, n, beta, digits, std = case
    sk = lwe_secret(variant, n, N, seed=51)
    z = rlwe_secret(N, seed=52)
    count = 5
    lwes = lwe_inputs(N, n, count, seed=53)
    accs = random_acc(N, count, seed=54)
    got = run(driver, tmp_path, "rotate", variant, N, n, beta, digits, std, 13, sk, z, lwes, count, accs)
    brk = oracle.br_keygen(variant, N, n, beta, digits, std, sk, z, seed=13)
    want = oracle.blind_rotate_many(variant, N, n, beta, digits, brk, lwes, accs, False, 2)
    assert np.array_equal(got.reshape(count, 2 * N), want)


@pytest.mark.gpu
def test_cpp_packer_like_oracle(driver, oracle, cuda, tmp_path):
    N, beta, digits, std, length = 128, 16, 4, 3.2, 4
    z = rlwe_secret(N, seed=61)
    lwes = (sm64(62, length * (N + 1)) % np.uint64(0xFFFFFFFF00000001)).reshape(length, N + 1)
    got = run(driver, tmp_path, "pack", N, beta, digits, std, 17, z, lwes, length)
    keys = oracle.pack_keygen(N, beta, digits, std, z, seed=17)
    want = oracle.pack(N, beta, digits, keys, lwes, length)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_cpp_sharded_pack_like_oracle(driver, oracle, cuda, tmp_path):
    """PackSubtree on each of W shards, then PackMerge over their roots: the words of one Pack."""
    N, beta, digits, std, length = 128, 16, 4, 3.2, 8
    z = rlwe_secret(N, seed=63)
    lwes = (sm64(64, length * (N + 1)) % np.uint64(0xFFFFFFFF00000001)).reshape(length, N + 1)
    keys = oracle.pack_keygen(N, beta, digits, std, z, seed=19)
    want = oracle.pack(N, beta, digits, keys, lwes, length)
    for shards in (2, 4):
        got = run(driver, tmp_path, "pack-shards", N, beta, digits, std, 19, z, lwes, length, shards)
        assert np.array_equal(got, want), shards


@pytest.mark.gpu
def test_cpp_function_evaluator_like_oracle(driver, oracle, cuda, tmp_path):
    """GpuNegacyclicFunctionEvaluator: BlindRotate (coefficient output) + SampleExtract into a
    caller buffer whose words stay where the rotated A coefficient is 0, as in the reference."""
    from oracle.oracle import P, ptr
    N, n, beta, digits = 256, 12, 16, 4
    sk = lwe_secret(CGGI_BINARY, n, N, seed=71)
    z = rlwe_secret(N, seed=72)
    lwes = lwe_inputs(N, n, 3, seed=73)
    lut = random_acc(N, 1, seed=74)[0]
    lut[:N] = 0                                        # trivial RLWE of a test polynomial
    lut[N + 5] = 0                                     # and a zero coefficient
    got = run(driver, tmp_path, "evalfunc", N, n, beta, digits, 19, sk, z, lwes, lut).reshape(3, N + 1)
    brk = oracle.br_keygen(CGGI_BINARY, N, n, beta, digits, 3.2, sk, z, seed=19)
    f_rlwe = np.zeros(2 * N, np.uint64)
    f_rlwe[0] = 1                                      # f(0) = 1 placed at A[0], as the reference does
    for i in range(1, N):
        f_rlwe[i + N] = (P - (3 * (N - i) + 1) % 5) % P
    for row, acc in ((0, lut), (1, f_rlwe), (2, lut)):
        rl = oracle.blind_rotate(CGGI_BINARY, N, n, beta, digits, brk, lwes[row], acc, 1)
        want = np.full(N + 1, 7, np.uint64)
        oracle.L.tpo_sample_extract(ptr(want), ptr(rl), 0, N)
        np.testing.assert_array_equal(got[row], want, err_msg=f"row {row}")


SS_CASE = (CGGI_BINARY, 256, 16, (16, 4), (14, 4), (20, 3), 3.2)


def test_scheme_switch_keygen_equals_oracle(driver, oracle, tmp_path):
    """keygen::SchemeSwitchingKeys draws the three keys from one stream in the reference's order."""
    variant, N, n, br, tr, sq, std = SS_CASE
    sk = lwe_secret(variant, n, N, seed=81)
    z = rlwe_secret(N, seed=82)
    got = run(driver, tmp_path, "keygen-ss", variant, N, n, *br, *tr, *sq, std, 23, sk, z)
    want = np.concatenate(oracle.ss_keygen(variant, N, n, br, tr, sq, std, sk, z, 23))
    assert np.array_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [CGGI_BINARY, BMMP_BINARY], ids=["cggi", "bmmp"])
def test_cpp_scheme_switch_like_oracle(driver, oracle, cuda, tmp_path, variant):
    _, N, n, br, tr, sq, std = SS_CASE
    D, ob, count = 4, 10, 3
    sk = lwe_secret(variant, n, N, seed=91)
    z = rlwe_secret(N, seed=92)
    lwes = lwe_inputs(N, n, count, seed=93)
    got = run(driver, tmp_path, "ss", variant, N, n, *br, *tr, *sq, std, 29, D, ob, sk, z, lwes, count)
    keys = oracle.ss_keygen(variant, N, n, br, tr, sq, std, sk, z, 29)
    for j in range(count):
        want = oracle.lwe_to_rgsw(variant, N, n, br, keys[0], tr, keys[1], sq, keys[2], D, ob, lwes[j])
        np.testing.assert_array_equal(got.reshape(count, -1)[j], want, err_msg=f"input {j}")


SAP_CASE = (CGGI_BINARY, 256, 10, (16, 4), (14, 4), (12, 5), 3.2)


def test_sap_keygen_equals_oracle(driver, oracle, tmp_path):
    """keygen::SAPKeys: rotation key, trace keys and the LWE key switch N -> n from one stream."""
    variant, N, n, br, tr, ks, std = SAP_CASE
    sk = lwe_secret(variant, n, N, seed=101)
    z = rlwe_secret(N, seed=102)
    got = run(driver, tmp_path, "keygen-sap", variant, N, n, *br, *tr, *ks, std, 31, sk, z)
    want = np.concatenate(oracle.sap_keygen(variant, N, n, br, tr, ks, std, sk, z, 31))
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_cpp_sap_like_oracle(driver, oracle, cuda, tmp_path):
    variant, N, n, br, tr, ks, std = SAP_CASE
    radix, restart, count, od = 4, 3, 3, 10
    sk = lwe_secret(variant, n, N, seed=111)
    z = rlwe_secret(N, seed=112)
    rng = np.random.default_rng(113)
    lwes = rng.integers(0, 1 << 16, (count, n + 1), dtype=np.uint64)
    lwes[1] &= np.uint64(0xFF)
    got = run(driver, tmp_path, "sap", variant, N, n, *br, *tr, *ks, std, 37, radix, restart, sk, z, lwes, count,
              od).reshape(count, od, N + 1)
    keys = oracle.sap_keygen(variant, N, n, br, tr, ks, std, sk, z, 37)
    beta = int(np.count_nonzero(sk))
    for j in range(count):
        _, want = oracle.sap_decompose(variant, N, n, br, keys[0], tr, keys[1], ks, keys[2], radix, beta, restart,
                                       lwes[j], od)
        np.testing.assert_array_equal(got[j], want, err_msg=f"input {j}")
