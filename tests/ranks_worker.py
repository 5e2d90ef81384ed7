"""One rank of tests/test_ranks.py (run as a script, RANK / WORLD_SIZE /
MASTER_ADDR / MASTER_PORT in the environment): gloo on the CPU, the helpers of
swb200.ranks, and a batch sharded over the ranks and aligned with the oracle."""
import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "projekt-2012_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import torch.distributed as dist  # noqa: E402

import oracle_ctypes as O  # noqa: E402
from swb200.ranks import gather_in_order, lpt_shards, max_over_ranks, replica_throughput  # noqa: E402


def batch(seed, n):
    rng = random.Random(seed)
    pairs = []
    for _ in range(n):
        la, lb = rng.randint(1, 300), rng.randint(0, 300)
        a = bytes(rng.choice(b"ACGT") for _ in range(la))
        b = a[rng.randint(0, la // 2):][:lb] + bytes(rng.choice(b"ACGT") for _ in range(rng.randint(0, 40)))
        pairs.append((a, b))
    return pairs


def align(pair, sc):
    rows, cols, swapped = O.orient(*pair)
    if not cols:
        return (0, 0, 0, swapped)
    e = O.stage1(rows, cols, O.scoring(*sc), O.TEXTBOOK, O.TIE_REFERENCE)
    return (e.score, e.row, e.col, swapped)


def main():
    out_path = sys.argv[1]
    dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=60))
    rank, world = dist.get_rank(), dist.get_world_size()
    # slowest rank's time, whole-job rate of the replicas
    ms = max_over_ranks(10.0 + 5.0 * rank, "cpu")
    assert ms == 10.0 + 5.0 * (world - 1), ms
    assert abs(replica_throughput(world, 1e6, 2, ms) - world * 2e6 / (ms * 1e-3)) < 1e-6
    # a batch sharded by cell count, aligned per rank, gathered in order
    sc = (2, -3, -5, -2)
    pairs = batch(5, 60)
    weights = [len(a) * len(b) for a, b in pairs]
    shards = lpt_shards(weights, world)
    mine = shards[rank]
    local = [align(pairs[i], sc) for i in mine]
    got = gather_in_order(local, mine, len(pairs))
    dist.barrier()
    if rank == 0:
        with open(out_path, "w") as f:
            json.dump({"results": got, "shards": shards,
                       "loads": [sum(weights[i] for i in s) for s in shards]}, f)
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
