"""One rank of the CPU multi-rank test (launched by torchrun with the gloo backend).

Follows the benchmark's multi-GPU plan on the oracle: every rank rotates its own
weak-scaling batch (seeds offset by rank), no collective touches the data, the
ranks' times are max-reduced, and rank 0 reports the whole-job rate. The ranks
gather the hashes of their outputs so the test can check each shard.
"""
import argparse
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from fhetoothpaste_b200.dist_util import aggregate_rate, env_ranks, init, max_over_ranks, weak_seed  # noqa: E402
from oracle.oracle import Oracle, lwe_inputs, lwe_secret, random_acc, rlwe_secret, sha256  # noqa: E402

SHAPE = (0, 128, 8, 16, 3)  # CGGI binary, N, n, beta, digits
PER_RANK = 3


def shard_outputs(oracle, rank):
    variant, N, n, beta, digits = SHAPE
    brk = oracle.br_keygen(variant, N, n, beta, digits, 3.2, lwe_secret(variant, n, N, 1), rlwe_secret(N, 2), 3)
    lwes = lwe_inputs(N, n, PER_RANK, weak_seed(7, rank))
    accs = random_acc(N, PER_RANK, weak_seed(8, rank))
    return oracle.blind_rotate_many(variant, N, n, beta, digits, brk, lwes, accs, False, 1)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    args = ap.parse_args()
    dist = init("gloo", timeout_s=60.0)
    rank, world, _ = env_ranks()
    assert dist is not None and dist.get_world_size() == world == 2
    out = shard_outputs(Oracle(), rank)
    seconds = 0.25 * (rank + 1)  # planted per-rank step times: the slowest rank is the last
    slowest = max_over_ranks(seconds, dist, "cpu")
    hashes = [None] * world
    dist.all_gather_object(hashes, (rank, sha256(out)))
    if rank == 0:
        Path(args.out).write_text(json.dumps({"slowest": slowest, "hashes": hashes,
                                              "rate": aggregate_rate(PER_RANK, world, slowest)}))
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
