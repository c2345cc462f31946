"""Batched NTT kernels against the reference's SolinasWorker outputs and the oracle."""
import numpy as np
import pytest

from oracle.oracle import P, uniform_mod

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("logn", range(7, 13))
def test_ntt_matches_reference(native, golden, cuda, logn):
    from fhetoothpaste_b200 import ntt_backward, ntt_forward
    torch = cuda
    manifest, arrays = golden
    N = 1 << logn
    x = uniform_mod(manifest["ntt"][str(N)]["seed"], N, P)
    d_in = torch.from_numpy(x.view(np.int64)).cuda()
    d_out = torch.empty_like(d_in)
    ntt_forward(N, 1, d_out.data_ptr(), d_in.data_ptr())
    np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint64), arrays[f"ntt_fwd_{N}"])
    ntt_backward(N, 1, d_out.data_ptr(), d_in.data_ptr())
    np.testing.assert_array_equal(d_out.cpu().numpy().view(np.uint64), arrays[f"ntt_bwd_{N}"])


@pytest.mark.parametrize("logn", [7, 10, 11, 12])
def test_ntt_batch_in_place_round_trip(native, oracle, cuda, logn):
    from fhetoothpaste_b200 import ntt_backward, ntt_forward
    torch = cuda
    N = 1 << logn
    count = 1500  # more polynomials than resident blocks
    x = uniform_mod(5 + logn, count * N, P).reshape(count, N)
    d = torch.from_numpy(x.view(np.int64)).cuda()
    ntt_forward(N, count, d.data_ptr(), d.data_ptr())
    f = d.cpu().numpy().view(np.uint64)
    for i in (0, 777, count - 1):
        np.testing.assert_array_equal(f[i], oracle.ntt_forward(x[i]))
    ntt_backward(N, count, d.data_ptr(), d.data_ptr())
    np.testing.assert_array_equal(d.cpu().numpy().view(np.uint64), x)


def test_sample_extract_matches_oracle(native, oracle, cuda):
    from fhetoothpaste_b200 import sample_extract_batch
    torch = cuda
    N, batch = 1024, 7
    r = uniform_mod(3, batch * 2 * N, P).reshape(batch, 2 * N)
    r[0, 5] = 0  # a zero coefficient: the reference leaves the (pre-zeroed) word alone
    d_in = torch.from_numpy(r.view(np.int64)).cuda()
    d_out = torch.empty((batch, N + 1), dtype=torch.int64, device="cuda")
    sample_extract_batch(N, batch, d_out.data_ptr(), d_in.data_ptr())
    got = d_out.cpu().numpy().view(np.uint64)
    for b in range(batch):
        exp = np.zeros(N + 1, np.uint64)
        oracle.L.tpo_sample_extract(exp.ctypes.data_as(oracle.L.tpo_sample_extract.argtypes[0]),
                                    np.ascontiguousarray(r[b]).ctypes.data_as(oracle.L.tpo_sample_extract.argtypes[1]),
                                    0, N)
        np.testing.assert_array_equal(got[b], exp)
