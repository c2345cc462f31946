"""Full-size checks on the benchmark's own workload (CGGI ternary n=630, N=2048, base 2^12
l=3, 4096 ciphertexts with their own test polynomials): ciphertexts sampled across the
persistent grid's waves equal the oracle; the batch is order-independent (a permuted batch
gives the permuted results, word for word); the two- and four-block kernels and a graph
replay give the one-block kernel's words."""
import numpy as np
import pytest

from oracle.oracle import CGGI_TERNARY, lwe_inputs, lwe_secret, random_acc, rlwe_secret

pytestmark = pytest.mark.gpu
N, n, BETA, L, BATCH = 2048, 630, 12, 3, 4096


@pytest.fixture(scope="module")
def setup(oracle):
    from fhetoothpaste_b200 import BlindRotationContext, GpuBlindRotator
    brk = oracle.br_keygen(CGGI_TERNARY, N, n, BETA, L, 3.2, lwe_secret(CGGI_TERNARY, n, N, 201),
                           rlwe_secret(N, 202), 203)
    rot = GpuBlindRotator(BlindRotationContext(CGGI_TERNARY, N, n, 1 << BETA, L), brk)
    lwes = lwe_inputs(N, n, BATCH, 204)
    accs = random_acc(N, BATCH, 205)
    out = rot.blind_rotate_batch_host(lwes, accs)
    return rot, brk, lwes, accs, out


def test_sampled_ciphertexts_equal_oracle(native, oracle, cuda, setup):
    rot, brk, lwes, accs, out = setup
    idx = [0, 147, 148, 295, 2048, 4095 - 148, 4094, 4095]  # wave boundaries of the 148-block grid
    want = oracle.blind_rotate_many(CGGI_TERNARY, N, n, BETA, L, brk, lwes[idx], accs[idx], False, 8)
    np.testing.assert_array_equal(out[idx], want)


def test_batch_order_does_not_matter(native, cuda, setup):
    rot, _, lwes, accs, out = setup
    perm = np.random.default_rng(206).permutation(BATCH)
    np.testing.assert_array_equal(rot.blind_rotate_batch_host(lwes[perm], accs[perm]), out[perm])


def test_row_by_row_form_gives_the_same_words(native, cuda, setup):
    rot, _, lwes, accs, out = setup
    assert rot.mac_form == 1
    rot.set_mac_form(0)
    try:
        np.testing.assert_array_equal(rot.blind_rotate_batch_host(lwes[:600], accs[:600]), out[:600])
    finally:
        rot.set_mac_form(1)


def test_two_blocks_and_graph_give_the_same_words(native, cuda, setup):
    torch = cuda
    rot, _, lwes, accs, out = setup
    for split, count in ((2, 300), (4, 100)):
        rot.set_split(split)
        try:
            np.testing.assert_array_equal(rot.blind_rotate_batch_host(lwes[:count], accs[:count]), out[:count],
                                          err_msg=f"{split} blocks per rotation")
        finally:
            rot.set_split(1)
    d_lwe = torch.from_numpy(lwes.view(np.int64)).cuda()
    d_acc = torch.from_numpy(accs.view(np.int64)).cuda()
    d_out = torch.empty((BATCH, 2 * N), dtype=torch.int64, device="cuda")
    g = rot.capture_batch(d_out.data_ptr(), d_lwe.data_ptr(), n + 1, d_acc.data_ptr(), 2 * N, BATCH)
    g.launch()
    rot.check()
    g.close()
    np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint64), out)
