"""The C oracle against golden vectors recorded from the reference library.

These pin the oracle: every GPU parity test compares against it.
"""
import numpy as np
import pytest

from brcases import case_inputs, case_key
from oracle.oracle import P, sha256, uniform_mod


@pytest.mark.parametrize("logn", range(7, 13))
def test_ntt_matches_reference(oracle, golden, logn):
    manifest, arrays = golden
    N = 1 << logn
    meta = manifest["ntt"][str(N)]
    x = uniform_mod(meta["seed"], N, P)
    assert sha256(x) == meta["input_sha256"]
    np.testing.assert_array_equal(oracle.ntt_forward(x), arrays[f"ntt_fwd_{N}"])
    np.testing.assert_array_equal(oracle.ntt_backward(x), arrays[f"ntt_bwd_{N}"])


def test_ntt_round_trip_and_monomial_order(oracle):
    # NTT(X^a)[k] = psi^((2 brv(k) + 1) a): the slot order every kernel relies on.
    N, logn = 256, 8
    psi = oracle.L.tpo_psi(N)
    a = 37
    x = np.zeros(N, np.uint64)
    x[a] = 1
    f = oracle.ntt_forward(x)
    for k in (0, 1, 5, 200):
        e = (2 * int(format(k, f"0{logn}b")[::-1], 2) + 1) * a % (2 * N)
        assert int(f[k]) == pow(psi, e, P)
    np.testing.assert_array_equal(oracle.ntt_backward(f), x)


@pytest.mark.parametrize("name", ["small_binary_n256", "small_ternary_n128", "small_bmmp_n512",
                                  "cfg1_binary_n1024", "cfg5a_ternary_n1024", "cfg2_ternary_n2048",
                                  "cfg3_bmmp_n2048", "cfg5c_ternary_n4096"])
def test_blind_rotate_matches_reference(oracle, golden, name):
    manifest, arrays = golden
    case = manifest["br"][name]
    _, _, brk = case_key(oracle, name, case)
    assert brk.size == case["key_words"]
    assert sha256(brk) == case["key_sha256"], "oracle key generation differs from the reference's"
    lwes, accs, coefs = case_inputs(name, case)
    expect = arrays[f"br_{name}"]
    for i, oc in enumerate(coefs):
        got = oracle.blind_rotate(case["variant"], case["N"], case["n"], case["basis_log2"], case["digits"],
                                  brk, lwes[i], accs[i], oc)
        np.testing.assert_array_equal(got, expect[i])
