"""The reference-side adapter (fhetoothpaste_b200/host/reference_adapter.hpp) under the
reference's own, unchanged callers of BlindRotator.

tests/cpp/reference_adapter_driver.cpp (built by oracle/Makefile into
oracle/_ref/libtpref_adapter.so, against the reference compiled from its own sources) runs each
caller twice with keys from the same sampler seed: over the reference's CPU rotator, wired as the
reference's tests wire it, and over toothpaste_b200::GpuRotationContext, an
OperatorContext<BlindRotator> whose operator rotates on the GPU. The outputs must be equal word
for word:
  - LWEtoRGSWConverter::Convert (lwe_to_rgsw_conversion.cpp:168-225),
  - SAPDecomposer::Decompose (sap_decomposer.cpp:353-464, rotations with result == accumulator),
  - BlindRotator::BlindRotate itself with result == accumulator, with coefficient output (the
    rotation NegacyclicFunctionEvaluator::EvalFunc makes, negacyclic_function_evaluator.cpp:92-101;
    the reference's evaluator itself cannot be constructed over a CGGI or BMMP context: its
    constructor dereferences a null container cast, lines 64-66) and NTT-domain output.
"""
import ctypes
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import (BMMP_BINARY, CGGI_BINARY, CGGI_TERNARY, P, lwe_inputs, lwe_secret, random_acc,
                           rlwe_secret)

ROOT = Path(__file__).resolve().parents[1]
LIB = ROOT / "oracle" / "_ref" / "libtpref_adapter.so"
U64P = ctypes.POINTER(ctypes.c_uint64)
U64, I32, F64 = ctypes.c_uint64, ctypes.c_int, ctypes.c_double


def _ptr(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(U64P)


@pytest.fixture(scope="module")
def adapter():
    if not LIB.exists():
        pytest.fail(f"{LIB} is missing: build it with `make -C oracle` (needs the reference sources once)")
    L = ctypes.CDLL(str(LIB))
    L.adp_last_error.restype = ctypes.c_char_p
    L.adp_lwe_to_rgsw.argtypes = [I32, U64, U64, U64, U64, U64, U64, U64, U64, F64, U64, U64, U64P, U64P, U64, U64,
                                  U64P, U64P, U64P]
    L.adp_sap.argtypes = [I32, U64, U64, U64, U64, U64, U64, U64, U64, F64, U64, U64P, U64P, U64, U64, U64P, U64,
                          U64P, U64P]
    L.adp_rotate_in_place.argtypes = [I32, U64, U64, U64, U64, F64, U64P, U64P, U64, U64, U64P, U64P, U64P, I32]
    return L


def _check(L, rc):
    assert rc == 0, L.adp_last_error().decode()


def test_adapter_library_exports_its_entry_points():
    """CPU: the adapter builds against the reference's headers and links both libraries."""
    if not LIB.exists():
        pytest.skip("adapter not built (reference sources absent when the oracle was built)")
    L = ctypes.CDLL(str(LIB))
    for name in ("adp_lwe_to_rgsw", "adp_sap", "adp_rotate_in_place", "adp_last_error"):
        assert hasattr(L, name), name


@pytest.mark.gpu
@pytest.mark.parametrize("variant,N,n,br,tr,sq,D,ob", [
    (CGGI_BINARY, 256, 16, (16, 4), (16, 4), (16, 4), 4, 16),
    (BMMP_BINARY, 256, 16, (12, 5), (14, 4), (20, 3), 4, 10),
    (CGGI_TERNARY, 128, 10, (16, 4), (14, 5), (16, 4), 2, 30)])
def test_lwe_to_rgsw_over_gpu_rotator(native, adapter, variant, N, n, br, tr, sq, D, ob):
    count = 2
    lk, rk = lwe_secret(variant, n, N, 21), rlwe_secret(N, 22)
    lwes = np.ascontiguousarray(lwe_inputs(N, n, count, 23))
    cpu = np.zeros((count, 4 * N * D), np.uint64)
    gpu = np.zeros((count, 4 * N * D), np.uint64)
    _check(adapter, adapter.adp_lwe_to_rgsw(variant, N, n, br[0], br[1], tr[0], tr[1], sq[0], sq[1], 3.2, D, ob,
                                            _ptr(lk), _ptr(rk), 24, count, _ptr(lwes), _ptr(cpu), _ptr(gpu)))
    assert np.any(cpu != 0)
    np.testing.assert_array_equal(gpu, cpu)


@pytest.mark.gpu
@pytest.mark.parametrize("variant,N,n,br,tr,ks,radix,bits", [
    (CGGI_BINARY, 256, 10, (16, 4), (16, 4), (16, 4), 4, 16),
    (CGGI_TERNARY, 256, 10, (12, 3), (16, 4), (16, 4), 4, 9)])
def test_sap_decomposer_over_gpu_rotator(native, adapter, variant, N, n, br, tr, ks, radix, bits):
    count = 2
    lk, rk = lwe_secret(variant, n, N, 31), rlwe_secret(N, 32)
    rng = np.random.default_rng(33)
    lwes = np.ascontiguousarray(rng.integers(0, 1 << bits, (count, n + 1), dtype=np.uint64))
    digits = -(-bits // (radix.bit_length() - 1)) + 1
    words = digits * (N + 1)
    cpu = np.zeros((count, words), np.uint64)
    gpu = np.zeros((count, words), np.uint64)
    _check(adapter, adapter.adp_sap(variant, N, n, br[0], br[1], tr[0], tr[1], ks[0], ks[1], 3.2, radix, _ptr(lk),
                                    _ptr(rk), 34, count, _ptr(lwes), words, _ptr(cpu), _ptr(gpu)))
    assert np.any(cpu != 0)
    np.testing.assert_array_equal(gpu, cpu)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [CGGI_BINARY, CGGI_TERNARY, BMMP_BINARY])
def test_blind_rotate_in_place_over_gpu_rotator(native, adapter, variant):
    N, n, bl, dg, count = 512, 24, 16, 4, 3
    lk, rk = lwe_secret(variant, n, N, 41), rlwe_secret(N, 42)
    lwes = np.ascontiguousarray(lwe_inputs(N, n, count, 43))
    for out_coef in (0, 1):
        cpu = np.ascontiguousarray(random_acc(N, count, 44))
        gpu = cpu.copy()
        _check(adapter, adapter.adp_rotate_in_place(variant, N, n, bl, dg, 3.2, _ptr(lk), _ptr(rk), 45, count,
                                                    _ptr(lwes), _ptr(cpu), _ptr(gpu), out_coef))
        assert np.all(cpu < P)
        np.testing.assert_array_equal(gpu, cpu)
