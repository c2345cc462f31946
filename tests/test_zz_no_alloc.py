"""The allocation-free packing entry point against the allocating one.

tp_pack_batch_noalloc exists for callers that cannot allocate device memory
when they call (their HBM belongs to another allocator's pool, or cudaMalloc's
blocking is unacceptable in their loop). It keeps its tree nodes in a fixed
16 MiB device array. Checked here through the C ABI: two calls in a row with
different inputs must each give exactly tp_pack_batch's result (the second after
a re-tiling of the context's key), and a call needing more than the fixed array,
or a pack count whose size wraps around 64 bits, must be refused.
"""
import ctypes

import numpy as np
import pytest

from kscases import ks_key
from oracle.oracle import P, uniform_mod

pytestmark = pytest.mark.gpu


def test_noalloc_pack_matches_allocating_pack(native, oracle, golden, cuda):
    from fhetoothpaste_b200 import _native
    torch = cuda
    name = "pack32_n256"
    c = golden[0]["ks"][name]
    N, bl, dg = c["N"], c["basis_log2"], c["digits"]
    keys = ks_key(oracle, name, c)
    h = ctypes.c_void_p()
    _native.check(native.tp_pack_create(N, 1 << bl, dg, 0, ctypes.byref(h)))
    try:
        _native.check(native.tp_ks_upload_key(h, _native.ptr(keys), keys.size))
        packs, length = 3, 32
        for call, seed in enumerate((101, 202)):
            if call == 1:
                # a re-tiling between the calls swaps the context's key buffer; the
                # call reads the new one under the context's lock
                _native.check(native.tp_ks_set_tile(h, 8 if native.tp_ks_get_tile(h) == 4 else 4))
            lwes = uniform_mod(seed, packs * length * (N + 1), P)
            d_in = torch.from_numpy(lwes.view(np.int64)).cuda()
            ref_out = torch.zeros((packs, 2 * N), dtype=torch.int64, device="cuda")
            got_out = torch.zeros((packs, 2 * N), dtype=torch.int64, device="cuda")
            _native.check(native.tp_pack_batch(h, packs, length, ref_out.data_ptr(), d_in.data_ptr(), None))
            _native.check(native.tp_pack_batch_noalloc(h, packs, length, got_out.data_ptr(), d_in.data_ptr(), None))
            torch.cuda.synchronize()
            np.testing.assert_array_equal(got_out.cpu().numpy(), ref_out.cpu().numpy(), err_msg=f"call {call}")

        # more than 2^21 words of nodes is refused, with a message
        too_many = (2 << 20) // (length * 2 * N) + 1
        st = native.tp_pack_batch_noalloc(h, too_many, length, got_out.data_ptr(), d_in.data_ptr(), None)
        assert st == _native.TP_ERR_PARAM
        assert b"fixed scratch" in native.tp_last_error()
        # a pack count whose word count wraps around 64 bits (2^50 * 32 * 2N = 2^64 at
        # N = 256) is refused too, not taken as a small call
        huge = 1 << 50
        st = native.tp_pack_batch_noalloc(h, huge, length, got_out.data_ptr(), d_in.data_ptr(), None)
        assert st == _native.TP_ERR_PARAM
        st = native.tp_pack_batch(h, huge, length, got_out.data_ptr(), d_in.data_ptr(), None)
        assert st == _native.TP_ERR_PARAM
        assert b"overflow" in native.tp_last_error()
    finally:
        native.tp_ks_destroy(h)
