"""The bootstrap epilogue on the GPU: FLOOR modulus switch, the fused SampleExtract -> LWE key
switch -> modulus switch (SAPDecomposer's refresh, lib/src/operators/sap_decomposer.cpp:353-369),
and whole bootstraps recorded as one graph, chained twice; bit-exact against the oracle, then
decrypted."""
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import CGGI_BINARY, P, lwe_encrypt_2n, lwe_secret, random_acc, rlwe_secret, sm64

pytestmark = pytest.mark.gpu
GOLD = Path(__file__).resolve().parent / "golden"


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.uint64).view(np.int64)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint64)


def test_modulus_switch_matches_reference(native, cuda):
    from fhetoothpaste_b200 import modulus_switch_batch
    d = np.load(GOLD / "modswitch.npz")
    for t in (256, 2048, 4096, 8192):
        for kind in ("round", "floor", "ceil"):
            x = dev(cuda, d[f"in_{t}"])
            modulus_switch_batch(x.numel(), x.data_ptr(), t, kind=kind)
            np.testing.assert_array_equal(host(x), d[f"{kind}_{t}"], err_msg=f"{kind} to {t}")


def test_modulus_switch_any_word_any_target(native, oracle, cuda):
    """Random words (some above p) and the neighbours of the rounding boundaries, targets 2 to 2^32,
    against the oracle's long-double switch."""
    from fhetoothpaste_b200 import modulus_switch_batch
    rng = np.random.default_rng(12)
    for k in (1, 5, 13, 20, 32):
        T = 1 << k
        xs = [int(v) for v in rng.integers(0, 2**64 - 1, 4000, dtype=np.uint64)] + [0, 1, P - 1, P, 2**64 - 1]
        for m in np.linspace(0, T - 1, 100).astype(np.int64).tolist():
            for base in ((m * P) // T, ((2 * m + 1) * P) // (2 * T)):
                xs += [base + d for d in range(-3, 4) if 0 <= base + d < 2**64]
        arr = np.array(xs, dtype=np.uint64)
        for kind in ("round", "floor", "ceil"):
            x = dev(cuda, arr)
            modulus_switch_batch(x.numel(), x.data_ptr(), T, kind=kind)
            np.testing.assert_array_equal(host(x), oracle.modulus_switch(arr, P, T, kind), err_msg=f"{kind} 2^{k}")


def test_modulus_switch_refuses_bad_arguments(native, cuda):
    from fhetoothpaste_b200 import _native
    x = cuda.zeros(4, dtype=cuda.int64, device="cuda")
    L = _native.lib()
    assert L.tp_modulus_switch_batch(4, x.data_ptr(), P, 2048, 3, None) == _native.TP_ERR_PARAM
    assert L.tp_modulus_switch_batch(4, x.data_ptr(), P, 3000, _native.TP_MS_FLOOR, None) == _native.TP_ERR_PARAM
    assert L.tp_modulus_switch_batch(4, x.data_ptr(), P - 2, 2048, _native.TP_MS_ROUND, None) == _native.TP_ERR_PARAM


def lut_value(f, k):
    """Coefficient 0 of f * X^k in Z_p[X]/(X^N + 1), 0 <= k < 2N (what SampleExtract reads)."""
    N = f.size
    sign, k = (1, k) if k < N else (-1, k - N)
    v = int(f[0]) if k == 0 else (P - int(f[N - k])) % P
    return v if sign > 0 else (P - v) % P


def ks_setup(oracle, N, n, beta, digits, seed):
    z = rlwe_secret(N, seed)                         # extracted-LWE key = RLWE key coefficients
    s = lwe_secret(CGGI_BINARY, n, N, seed + 1)      # target LWE key {0, 1}
    ksk = oracle.lwe_ks_keygen(P, N, n, beta, digits, 3.2, z, s, seed + 2)
    return z, s, ksk


@pytest.mark.parametrize("N,n", [(256, 32), (2048, 630)])
def test_epilogue_matches_oracle(native, oracle, cuda, N, n):
    from fhetoothpaste_b200 import GpuLWEtoLWEConverter
    beta, digits, batch = 16, 4, 37
    _, _, ksk = ks_setup(oracle, N, n, beta, digits, 300 + N)
    conv = GpuLWEtoLWEConverter(N, n, 1 << beta, digits, ksk)
    rl = random_acc(N, batch, 400 + N)
    d_in = dev(cuda, rl)
    d_out = cuda.full((batch, n + 1), -1, dtype=cuda.int64, device="cuda")  # written fresh, not accumulated
    for _ in range(2):
        conv.pbs_epilogue_batch(batch, d_out.data_ptr(), d_in.data_ptr(), 2 * N)
    got = host(d_out)
    for b in (0, batch // 2, batch - 1):
        np.testing.assert_array_equal(got[b], oracle.pbs_epilogue(rl[b], n, beta, digits, ksk, 2 * N))
    assert got.max() < 2 * N


def test_two_chained_bootstraps(native, oracle, cuda):
    """LWE (mod 2N) -> [rotation -> extract -> key switch -> switch to 2N] x 2 through one recorded graph
    per bootstrap; every stage equals the oracle and the output decrypts to the rotated test value."""
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator, GpuLWEtoLWEConverter
    N, n, beta, digits, batch = 1024, 64, 16, 4, 8
    z, s, ksk = ks_setup(oracle, N, n, beta, digits, 900)
    brk = oracle.br_keygen(CGGI_BINARY, N, n, beta, digits, 3.2, s, z, 903)
    rot = GpuBlindRotator(BlindRotationContext(CGGI_BINARY, N, n, 1 << beta, digits), brk)
    conv = GpuLWEtoLWEConverter(N, n, 1 << beta, digits, ksk)
    delta = P // 16
    f = np.array([((i * 16) // N) % 8 * delta for i in range(N)], dtype=np.uint64)  # 8 plateaus of N/8 = 128
    acc = np.concatenate([np.zeros(N, np.uint64), f])
    msgs = [int(m) * (2 * N // 16) + 64 for m in sm64(904, batch) % np.uint64(8)]
    lwe0 = lwe_encrypt_2n(s, N, msgs, 905)
    d_lwe = [dev(cuda, lwe0), cuda.empty((batch, n + 1), dtype=cuda.int64, device="cuda"),
             cuda.empty((batch, n + 1), dtype=cuda.int64, device="cuda")]
    d_acc = dev(cuda, acc)
    d_rl = cuda.empty((batch, 2 * N), dtype=cuda.int64, device="cuda")
    graphs = [rot.capture_bootstrap(conv, batch, d_rl.data_ptr(), d_lwe[k].data_ptr(), d_acc.data_ptr(), 0,
                                    d_lwe[k + 1].data_ptr()) for k in range(2)]
    want = lwe0
    s2n = s.astype(np.int64)
    for k in range(2):
        graphs[k].launch()
        rot.check()
        got = host(d_lwe[k + 1])
        exp = []
        for b in range(batch):
            rl = oracle.blind_rotate(CGGI_BINARY, N, n, beta, digits, brk, want[b], acc, 1)
            exp.append(oracle.pbs_epilogue(rl, n, beta, digits, ksk, 2 * N))
        exp = np.stack(exp)
        np.testing.assert_array_equal(got, exp, err_msg=f"bootstrap {k}")
        # decrypt: phase mod 2N is the test polynomial's value at the rotated position, scaled to 2N
        for b in range(batch):
            phase_in = (int(want[b][n]) - int(want[b][:n].astype(np.int64) @ s2n)) % (2 * N)
            value = lut_value(f, phase_in)
            expect = value * 2 * N // P
            phase_out = (int(got[b][n]) - int(got[b][:n].astype(np.int64) @ s2n)) % (2 * N)
            dist = min((phase_out - expect) % (2 * N), (expect - phase_out) % (2 * N))
            assert dist <= n // 2 + 4, (k, b, phase_in, phase_out, expect)
        want = got
    for g in graphs:
        g.close()
