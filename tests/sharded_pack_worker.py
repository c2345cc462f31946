"""One rank of the sharded-packing test (launched by torchrun with gloo, CPU only).

The two packing steps are stood in for by bookkeeping on leaf lists: a node is the list of
input indices on its leaves, in tree order (padded with -1), so the exchange order, the
shard rows and the level bookkeeping of fhetoothpaste_b200.sharded_pack are checked
against the reference tree's leaf order, (len - 1) ^ brv(c) on leaf c."""
import argparse
import json
import sys
from pathlib import Path

import numpy as np
import torch
import torch.distributed as dist

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from fhetoothpaste_b200.sharded_pack import _brv, pack_sharded, shard_inputs  # noqa: E402


def leaf_ops(length: int, log_n: int, calls: list):
    def subtree(inputs, m):
        packs = inputs.shape[0] // m
        out = torch.full((packs, length), -1, dtype=torch.int64)
        lb = m.bit_length() - 1
        for p in range(packs):
            for c in range(m):
                out[p, c] = inputs[p * m + ((m - 1) ^ _brv(c, lb)), 0]
        return out

    def merge(nodes, count, level0, finish):
        calls.append((count, level0, bool(finish)))
        packs = nodes.shape[0]
        out = torch.full((packs, length), -1, dtype=torch.int64)
        for p in range(packs):
            leaves = [int(v) for q in range(count) for v in nodes[p, q] if v >= 0]
            # every node of level L covers 2^L leaves
            assert all(int((nodes[p, q] >= 0).sum()) == 1 << level0 for q in range(count))
            out[p, :len(leaves)] = torch.tensor(leaves)
        assert finish == (level0 + (count.bit_length() - 1) == length.bit_length() - 1)
        return out

    return subtree, merge


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--length", type=int, default=16)
    ap.add_argument("--packs", type=int, default=3)
    a = ap.parse_args()
    dist.init_process_group("gloo")
    rank, world = dist.get_rank(), dist.get_world_size()
    length, packs = a.length, a.packs
    # input row e of pack p carries its global index p * length + e
    rows = np.arange(packs * length, dtype=np.int64).reshape(packs * length, 1)
    local = torch.from_numpy(shard_inputs(rows, packs, length, world, rank))
    calls = []
    subtree, merge = leaf_ops(length, 11, calls)
    root = pack_sharded(subtree, merge, local, packs, length, world, rank, dist)
    got = [[int(v) for v in root[p] if v >= 0] for p in range(packs)]
    lb = length.bit_length() - 1
    want = [[p * length + ((length - 1) ^ _brv(c, lb)) for c in range(length)] for p in range(packs)]
    rep = {"rank": rank, "ok": got == want, "calls": calls}
    reps = [None] * world
    dist.all_gather_object(reps, rep)
    if rank == 0:
        Path(a.out).write_text(json.dumps(reps))
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
