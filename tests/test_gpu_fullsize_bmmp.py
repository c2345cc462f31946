"""Full-size BMMP parity at the batch sizes of the benchmark's BMMP sweep (binary n=768 as 384
pairs, N=2048, base 2^16 l=4, identity test polynomial): batches of 2048 and 8192 ciphertexts,
ciphertexts sampled across the persistent grid's waves equal the oracle word for word, with the
digit-staged and the row-by-row multiply-accumulate."""
import numpy as np
import pytest

from oracle.oracle import BMMP_BINARY, lwe_inputs, lwe_secret, rlwe_secret

pytestmark = pytest.mark.gpu
N, n, BETA, L = 2048, 768, 16, 4


@pytest.fixture(scope="module")
def bmmp(oracle):
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    brk = oracle.br_keygen(BMMP_BINARY, N, n, BETA, L, 3.2, lwe_secret(BMMP_BINARY, n, N, 301),
                           rlwe_secret(N, 302), 303)
    rot = GpuBlindRotator(BlindRotationContext(BMMP_BINARY, N, n, 1 << BETA, L), brk)
    ident = np.zeros(2 * N, np.uint64)
    ident[N:] = np.arange(N, dtype=np.uint64)
    return rot, brk, ident


@pytest.mark.parametrize("batch", [2048, 8192])
def test_bmmp_large_batch_samples_equal_oracle(native, oracle, cuda, bmmp, batch):
    rot, brk, ident = bmmp
    lwes = lwe_inputs(N, n, batch, 304 + batch)
    idx = sorted({0, 147, 148, 295, batch // 2, batch - 149, batch - 1})
    want = oracle.blind_rotate_many(BMMP_BINARY, N, n, BETA, L, brk, lwes[idx],
                                    np.repeat(ident[None, :], len(idx), axis=0), False, 8)
    for form in (1, 0):
        rot.set_mac_form(form)
        got = rot.blind_rotate_batch_host(lwes, ident)
        np.testing.assert_array_equal(got[idx], want, err_msg=f"form {form}")
    rot.set_mac_form(1)
