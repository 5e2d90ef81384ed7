"""One rank of the column-chunk chain in tests/test_chain.py (run as a script,
RANK / WORLD_SIZE / MASTER_ADDR / MASTER_PORT in the environment): gloo on the
CPU, the oracle's block function standing in for the GPU's, borders passed by
point-to-point send/recv as on GPUs."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "projekt-2012_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)

import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

from swb200 import chain  # noqa: E402
from chain_cases import case, oracle_block  # noqa: E402


def main():
    out_path, seed, height, tie = sys.argv[1], int(sys.argv[2]), int(sys.argv[3]), int(sys.argv[4])
    dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=60))
    rank, world = dist.get_rank(), dist.get_world_size()
    rows, cols, sc = case(seed)
    blk = oracle_block(rows, cols, sc, tie, as_torch=True)
    send, recv = chain.torch_links()
    mine = chain.run_rank(rank, world, len(rows), len(cols), height, blk, send, recv)
    best = chain.gather_best(mine)
    if rank == 0:
        with open(out_path, "w") as f:
            json.dump({"best": list(best)}, f)
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
