"""LWEtoRLWEPacker::Pack (lib/src/operators/lwe_to_rlwe_packing.cpp:129-236) split over W
ranks, one GPU each: every rank packs one subtree of the tree, then the ranks combine
their roots with log2 W pairwise exchanges of one RLWE per pack.

The reference's tree puts input (len - 1) ^ brv_{log2 len}(c) on leaf c, and a merge at
tree level L depends only on L (automorphism key 2^L + 1, shift N >> L), not on where
the node sits. So the subtree of leaves [r m, (r + 1) m), m = len / W, is a pack of m
inputs, those with index j W + s, s = (W - 1) ^ brv_{log2 W}(r) (brv over log2 len bits
of r m + c' is brv(c') W + brv(r)). Rank r packs that subtree (tp_pack_subtree_batch);
at step k = 1 .. log2 W it swaps its current root with rank r ^ 2^(k-1) and both merge
the pair at level log2 m + k (the rank whose bit k-1 is clear holds the left node);
the last step also applies the trailing traces (tp_pack_merge_batch), so every rank ends
with the packed RLWE that a single-device Pack gives, word for word.

The exchange and the index arithmetic are written over two callables, so the same code
runs the GPU kernels (`gpu_packing_ops`) and any other implementation of the two steps.
"""
from __future__ import annotations

from typing import Callable

import numpy as np


def _log2(x: int) -> int:
    if x < 1 or x & (x - 1):
        raise ValueError(f"{x} is not a power of two")
    return x.bit_length() - 1


def _brv(x: int, bits: int) -> int:
    r = 0
    for b in range(bits):
        r |= ((x >> b) & 1) << (bits - 1 - b)
    return r


def shard_offset(world: int, rank: int) -> int:
    """s: rank `rank` packs the inputs j * world + s."""
    w = _log2(world)
    return (world - 1) ^ _brv(rank, w)


def shard_rows(length: int, world: int, rank: int) -> np.ndarray:
    """Row indices (within one pack of `length` inputs) of rank `rank`'s subtree, in the
    subtree's own input order."""
    if length % world or length < world:
        raise ValueError("the pack length must be a multiple of the number of ranks")
    _log2(length)
    return np.arange(length // world, dtype=np.int64) * world + shard_offset(world, rank)


def shard_inputs(lwes: np.ndarray, packs: int, length: int, world: int, rank: int) -> np.ndarray:
    """This rank's inputs: packs x (length / world) rows of N + 1 words."""
    x = np.asarray(lwes).reshape(packs, length, -1)
    return np.ascontiguousarray(x[:, shard_rows(length, world, rank), :]).reshape(packs * (length // world), -1)


def pack_sharded(subtree: Callable, merge: Callable, local_inputs, packs: int, length: int, world: int,
                 rank: int, dist=None):
    """Runs this rank's part of a sharded Pack and returns the packed RLWEs (packs x 2N).

    subtree(inputs, m) -> roots (packs x S): pack the m-input subtrees, no traces.
    merge(nodes, count, level0, finish) -> roots (packs x S): nodes is packs x count x S.
    dist: torch.distributed (None or world 1: one rank). Every rank calls the same
    collectives in the same order."""
    import torch
    w = _log2(world)
    m = length // world
    if m < 1 or m * world != length:
        raise ValueError("the pack length must be a multiple of the number of ranks")
    node = subtree(local_inputs, m)
    level = _log2(m)
    if w == 0:
        return merge(node.reshape(packs, 1, -1), 1, level, True)
    for k in range(1, w + 1):
        partner = rank ^ (1 << (k - 1))
        other = torch.empty_like(node)
        ops = [dist.P2POp(dist.isend, node.contiguous(), partner), dist.P2POp(dist.irecv, other, partner)]
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        left, right = (node, other) if (rank >> (k - 1)) & 1 == 0 else (other, node)
        pair = torch.stack([left, right], dim=1)                    # packs x 2 x S
        node = merge(pair, 2, level, k == w)
        level += 1
    return node


def gpu_packing_ops(packer, stream=None):
    """The two steps on a GpuLWEtoRLWEPacker, over int64 CUDA tensors of uint64 words."""
    import torch
    N = packer.N

    def subtree(inputs, m):
        packs = inputs.numel() // (m * (N + 1))
        out = torch.empty((packs, 2 * N), dtype=torch.int64, device=inputs.device)
        packer.pack_subtree_batch(packs, m, out.data_ptr(), inputs.contiguous().data_ptr(), stream)
        return out

    def merge(nodes, count, level0, finish):
        nodes = nodes.contiguous()
        packs = nodes.shape[0]
        out = torch.empty((packs, 2 * N), dtype=torch.int64, device=nodes.device)
        packer.pack_merge_batch(packs, count, level0, finish, out.data_ptr(), nodes.data_ptr(), stream)
        return out

    return subtree, merge
