"""The multi-GPU plan's host side on two CPU ranks (gloo, launched like the benchmark by torchrun):
per-rank weak-scaling shards, max-over-ranks timing, whole-job rate. No GPU involved."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np

from oracle.oracle import sha256

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "tests"))


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_shard_and_reduce(oracle, tmp_path):
    import multirank_worker as w
    out = tmp_path / "rank0.json"
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={free_port()}", str(ROOT / "tests" / "multirank_worker.py"),
           "--out", str(out)]
    res = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    rep = json.loads(out.read_text())
    assert rep["slowest"] == 0.5                                  # max of 0.25 and 0.5
    assert rep["rate"] == w.PER_RANK * 2 / 0.5                    # units of all ranks / slowest time
    by_rank = dict(rep["hashes"])
    assert sorted(by_rank) == [0, 1]
    for r in (0, 1):                                              # each shard = its rank's own batch
        assert by_rank[r] == sha256(w.shard_outputs(oracle, r))
    assert by_rank[0] != by_rank[1]                               # the ranks rotate different inputs


def test_single_process_needs_no_group():
    from fhetoothpaste_b200.dist_util import aggregate_rate, init, max_over_ranks
    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        assert init("gloo") is None
        assert max_over_ranks(1.5, None, "cpu") == 1.5
        assert aggregate_rate(4096, 1, 0.5) == 8192
    finally:
        os.environ.update(env)


def _run_sharded_pack(tmp_path, world: int, length: int):
    out = tmp_path / f"pack{world}.json"
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", CUDA_VISIBLE_DEVICES="")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={world}",
           "--master-addr=127.0.0.1", f"--master-port={free_port()}", str(ROOT / "tests" / "sharded_pack_worker.py"),
           "--out", str(out), "--length", str(length)]
    res = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    return json.loads(out.read_text())


def test_sharded_packing_exchange_on_two_and_four_ranks(tmp_path):
    """Pack split over W ranks (fhetoothpaste_b200/sharded_pack.py): each rank's shard rows, the
    log2 W pairwise exchanges and the merge levels give the reference tree's leaf order on every
    rank, with the traces applied once, on the last merge."""
    for world, length in ((2, 16), (4, 16), (4, 4)):
        reps = _run_sharded_pack(tmp_path, world, length)
        assert [r["rank"] for r in reps] == list(range(world))
        m = length // world
        for r in reps:
            assert r["ok"], (world, length, r)
            lm = m.bit_length() - 1
            w = world.bit_length() - 1
            assert r["calls"] == [[2, lm + k, k == w - 1] for k in range(w)]


def test_shard_rows_cover_every_input_once():
    from fhetoothpaste_b200.sharded_pack import shard_rows
    for length in (2, 8, 64, 2048):
        for world in (1, 2, 4, 8):
            if world > length:
                continue
            rows = np.concatenate([shard_rows(length, world, r) for r in range(world)])
            assert sorted(rows.tolist()) == list(range(length))
