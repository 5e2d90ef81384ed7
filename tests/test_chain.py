"""The multi-GPU column-chunk chain for one long pair (swb200/chain.py).

Runs with one GPU per process in production; the GPU tests get one GPU, so
the protocol is checked on the CPU: the oracle's block function (orc_block)
stands in for swb_score_block_device, in one process (virtual ranks) and as 2
and 3 gloo ranks in subprocesses exchanging borders by point-to-point
send/recv as NCCL would between GPUs.  Every chain gives the oracle's
whole-matrix score and end cell under both tie rules.  The GPU test drives
swb_score_block_device through the same protocol with virtual ranks on one GPU.
The multi-process NCCL path is not run on GPUs here (one GPU per run).
"""
import json
import os
import random
import socket
import subprocess
import sys

import numpy as np
import pytest

import oracle_ctypes as O
from chain_cases import case, oracle_block
from swb200 import chain

HERE = os.path.dirname(os.path.abspath(__file__))


def _whole(rows, cols, sc, tie):
    e = O.stage1(rows, cols, O.scoring(*sc), O.TEXTBOOK, tie)
    return e.score, e.row, e.col


def test_chunks_and_blocks():
    assert chain.column_chunks(1000, 1) == [(0, 1000)]
    ch = chain.column_chunks(10_000, 4)
    assert ch[0][0] == 0 and ch[-1][1] == 10_000
    assert all(a[1] == b[0] for a, b in zip(ch, ch[1:]))
    assert all(lo % 256 == 0 for lo, _ in ch)
    assert chain.row_blocks(1500, 512) == [(0, 512), (512, 1024), (1024, 1500)]
    with pytest.raises(ValueError):
        chain.row_blocks(1000, 500)
    assert chain.merge([(5, 1, 1, 9), (5, 2, 2, 3), (4, 0, 0, 0)]) == (5, 2, 2, 3)
    assert chain.merge([(0, 0, 0, chain.NO_KEY)]) == (0, 0, 0, chain.NO_KEY)


def test_single_block_equals_the_whole_matrix():
    rows, cols, sc = case(3)
    for tie in (O.TIE_REFERENCE, O.TIE_ROWMAJOR):
        _, _, e, key = O.block(rows, cols, O.scoring(*sc), None, None, 0, 0, 0, len(rows), len(cols), tie)
        assert (e.score, e.row, e.col) == _whole(rows, cols, sc, tie)


@pytest.mark.parametrize("seed", range(8))
def test_virtual_ranks_equal_the_whole_matrix(seed):
    rows, cols, sc = case(seed)
    rng = random.Random(seed)
    for tie in (O.TIE_REFERENCE, O.TIE_ROWMAJOR):
        world = rng.randint(1, 6)
        height = rng.choice([512, 1024])
        got = chain.run_virtual(world, len(rows), len(cols), height, oracle_block(rows, cols, sc, tie))
        assert got[:3] == _whole(rows, cols, sc, tie), (world, height)


def test_borders_match_the_whole_matrix_rows():
    """A block's bottom row and right column are the whole matrix's (H, F) and
    (H, E) there (special rows of the oracle give the row)."""
    rows, cols, sc = case(1)
    s = O.scoring(*sc)
    bottom, right, _, _ = O.block(rows[:1024], cols, s, None, None, 0, 0, 0, len(rows), len(cols), O.TIE_REFERENCE)
    ref = O.special_rows(rows[:1024], cols, s, 1024)[0]
    assert np.array_equal(bottom, ref)
    # the right border of the left half feeds the right half: chained result = whole
    half = (len(cols) // 2 // 256) * 256
    b1, r1, e1, k1 = O.block(rows[:1024], cols[:half], s, None, None, 0, 0, 0, len(rows), len(cols), O.TIE_REFERENCE)
    b2, r2, e2, k2 = O.block(rows[:1024], cols[half:], s, None, r1, 0, 0, half, len(rows), len(cols), O.TIE_REFERENCE)
    assert np.array_equal(np.concatenate([b1, b2]), ref)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,seed,height,tie", [(2, 4, 512, 0), (3, 5, 1024, 1), (3, 6, 512, 0)])
def test_gloo_ranks_equal_the_whole_matrix(tmp_path, world, seed, height, tie):
    out = str(tmp_path / "chain.json")
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "chain_worker.py"), out, str(seed),
                                       str(height), str(tie)], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.STDOUT))
    logs = []
    for p in procs:
        try:
            logs.append(p.communicate(timeout=180)[0].decode(errors="replace"))
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
    assert all(p.returncode == 0 for p in procs), logs
    got = tuple(json.load(open(out))["best"])
    rows, cols, sc = case(seed)
    assert got[:3] == _whole(rows, cols, sc, tie)


@pytest.mark.gpu
@pytest.mark.parametrize("world,height", [(3, 512), (4, 1024)])
def test_gpu_blocks_through_the_chain(world, height):
    """swb_score_block_device as the block function of the chain (virtual ranks
    on one GPU): the oracle's whole-matrix result under both tie rules, and the
    borders of a block equal the oracle's."""
    import torch
    import swb200
    for seed in (1, 2):
        rows, cols, sc_t = case(seed + 10 * world)
        for tie in (0, 1):
            with swb200.Context(device=0) as ctx:
                d_rows = torch.frombuffer(bytearray(rows), dtype=torch.uint8).cuda()
                d_cols = torch.frombuffer(bytearray(cols), dtype=torch.uint8).cuda()
                blk = chain.GpuBlocks(ctx, d_rows, d_cols, swb200.scoring(*sc_t),
                                      swb200.FLAG_TIE_ROWMAJOR if tie else 0)
                got = chain.run_virtual(world, len(rows), len(cols), height, blk)
                assert got[:3] == _whole(rows, cols, sc_t, tie), (seed, tie)
                # one interior block's borders against the oracle's
                r_lo, c_lo = height, (len(cols) // 2 // 256) * 256
                r_hi, c_hi = min(len(rows), r_lo + height), len(cols)
                if r_hi - r_lo == height and c_lo > 0:
                    s = O.scoring(*sc_t)
                    # the left border comes from the whole-matrix rows r_lo.. of column c_lo - 1
                    _, left_b, _, _ = O.block(rows[:r_hi], cols[:c_lo], s, None, None, 0, 0, 0, len(rows),
                                              len(cols), tie)
                    left_b = left_b[r_lo:r_hi]
                    h_up = O.special_rows(rows[:r_lo], cols[:c_lo], s, r_lo)[0]
                    corner = int(h_up[c_lo - 1][0])
                    top_full = O.special_rows(rows[:r_lo], cols, s, r_lo)[0][c_lo:]
                    exp_bottom, exp_right, e, key = O.block(rows[r_lo:r_hi], cols[c_lo:], s, top_full, left_b,
                                                            corner, r_lo, c_lo, len(rows), len(cols), tie)
                    d_top = torch.from_numpy(np.ascontiguousarray(top_full)).cuda()
                    d_left = torch.from_numpy(np.ascontiguousarray(left_b)).cuda()
                    bottom, right, best = blk(r_lo, r_hi, c_lo, c_hi, d_top, d_left, corner, True, True)
                    assert np.array_equal(bottom.cpu().numpy(), exp_bottom)
                    assert np.array_equal(right.cpu().numpy(), exp_right)
                    assert best[:3] == ((e.score, e.row, e.col) if e.score > 0 else (0, -1, -1))
