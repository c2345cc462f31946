"""A packing split into subtrees (tp_pack_subtree_batch) and merged above them
(tp_pack_merge_batch), the two steps of the multi-GPU packing in
fhetoothpaste_b200/sharded_pack.py, run here on one GPU for W = 1 .. 16 shards: the
same words as one Pack, against the reference's golden outputs and the oracle."""
import json
from pathlib import Path

import numpy as np
import pytest

from kscases import ks_inputs, ks_key
from oracle.oracle import P, sha256, uniform_mod

pytestmark = pytest.mark.gpu


def _emulate(packer, lwes, packs, length, world, pairwise=True):
    """Every shard's subtree, then the pairwise merges the ranks of pack_sharded make
    (or one merge of all roots), in one process."""
    import torch
    from fhetoothpaste_b200.sharded_pack import gpu_packing_ops, shard_inputs
    subtree, merge = gpu_packing_ops(packer)
    m = length // world
    nodes = [subtree(torch.from_numpy(shard_inputs(lwes, packs, length, world, r).view(np.int64)).cuda(), m)
             for r in range(world)]
    level = m.bit_length() - 1
    if world == 1:
        root = merge(nodes[0].reshape(packs, 1, -1), 1, level, True)
    elif pairwise:
        while len(nodes) > 1:
            last = len(nodes) == 2
            nodes = [merge(torch.stack([nodes[2 * i], nodes[2 * i + 1]], dim=1), 2, level, last)
                     for i in range(len(nodes) // 2)]
            level += 1
        root = nodes[0]
    else:
        root = merge(torch.stack(nodes, dim=1), world, level, True)
    return root.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("world", [1, 2, 8, 16])
def test_sharded_pack_matches_reference_n2048(native, oracle, golden, world):
    from fhetoothpaste_b200 import GpuLWEtoRLWEPacker
    name = "pack2048_n2048"
    c, expect = golden[0]["ks"][name], golden[1][f"ks_{name}"]
    pk = GpuLWEtoRLWEPacker(c["N"], 1 << c["basis_log2"], c["digits"], ks_key(oracle, name, c))
    x = ks_inputs(c)
    np.testing.assert_array_equal(_emulate(pk, x, 1, c["len"], world)[0], expect[0])
    if world > 2:
        np.testing.assert_array_equal(_emulate(pk, x, 1, c["len"], world, pairwise=False)[0], expect[0])
    pk.close()


def test_sharded_pack_many_packs_short_lengths(native, oracle, golden):
    """Several packs per call, trailing traces after the top merge, and shards of one input."""
    from fhetoothpaste_b200 import GpuLWEtoRLWEPacker
    name = "pack32_n256"
    c = golden[0]["ks"][name]
    N, k = c["N"], ks_key(oracle, name, c)
    pk = GpuLWEtoRLWEPacker(N, 1 << c["basis_log2"], c["digits"], k)
    packs = 3
    for length, world in ((16, 4), (8, 8), (4, 2)):
        lwes = uniform_mod(70 + length, packs * length * (N + 1), P).reshape(packs * length, N + 1)
        whole = pk.Pack(lwes, length)
        got = _emulate(pk, lwes, packs, length, world)
        np.testing.assert_array_equal(got, whole, err_msg=f"len {length}, {world} shards")
        exp = oracle.pack(N, c["basis_log2"], c["digits"], k, lwes[length:2 * length], length)
        np.testing.assert_array_equal(got[1], exp)
    pk.close()


def test_sharded_pack_matches_reference_n8192(native, oracle):
    """Ring size 8192 (cluster kernels), the reference's own output."""
    from fhetoothpaste_b200 import GpuLWEtoRLWEPacker
    name = "pack16_n8192"
    c = json.loads((Path(__file__).resolve().parent / "golden" / "largen.json").read_text())["ks"][name]
    pk = GpuLWEtoRLWEPacker(c["N"], 1 << c["basis_log2"], c["digits"], ks_key(oracle, name, c))
    got = _emulate(pk, ks_inputs(c), 1, c["len"], 4)
    assert sha256(np.ascontiguousarray(got[0])) == c["out_sha256"][0]
    pk.close()


def test_shard_arguments_are_checked(native, oracle, golden):
    from fhetoothpaste_b200 import GpuLWEtoRLWEPacker, _native
    name = "pack32_n256"
    c = golden[0]["ks"][name]
    pk = GpuLWEtoRLWEPacker(c["N"], 1 << c["basis_log2"], c["digits"], ks_key(oracle, name, c))
    with pytest.raises(_native.TpError):
        pk.pack_subtree_batch(1, 3, 16, 16)                 # length not a power of two
    with pytest.raises(_native.TpError):
        pk.pack_merge_batch(1, 4, 7, True, 16, 16)          # level 7 + 2 above log2 N = 8
    with pytest.raises(_native.TpError):
        pk.pack_merge_batch(1, 3, 0, True, 16, 16)          # count not a power of two
    pk.close()
