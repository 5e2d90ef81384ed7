"""The multi-GPU chain for one long pair: the pair's columns are cut into one
chunk per GPU, and each GPU walks its chunk in blocks of rows.

The reference aligns one pair on one GPU (src/main.cu:125-126).  Past one B200
the pair's anti-diagonal wavefront continues across GPUs in column chunks:

* rank g owns columns [C_g, C_{g+1}) (inner boundaries at multiples of 256) and
  walks row blocks [R_b, R_{b+1}) in order (heights a multiple of 512 rows, so
  the block's last row is a strip bottom of the scoring kernel);
* block b of rank g starts from the bottom row of its own block b-1 (top
  boundary, (H, F) per column), the right border of block b of rank g-1 (left
  boundary, (H, E) per row) and the corner H[R_b - 1][C_g - 1], which is the last
  row of the left border received for block b-1;
* it sends its own right border to rank g+1: a point-to-point transfer into the
  receiver's own buffer (torch.distributed send/recv: NCCL over NVLink between
  GPUs, gloo on the CPU), no collective and no multicast on the data path;
* each block reports its best cell in whole-matrix coordinates with the
  reference's tie key over the whole matrix, so after the last block the ranks
  merge their candidates (highest score, then smallest key) into the pair's
  result, the same score and end cell one GPU gives.

Rank g runs block b while rank g-1 runs block b+1, so with B row blocks the
chain is busy for B + world - 1 block times; blocks of about a million rows
keep every warp of a B200 busy inside each block (a million rows are about
2,200 strips of 448 rows, against 2,368 resident warps).

The protocol is written against three callables so that the same code runs
with the GPU (GpuBlocks below, one process per GPU, NCCL) and with the CPU
oracle in tests (gloo):
  block(r_lo, r_hi, c_lo, c_hi, top, left, corner, want_bottom, want_right)
      -> (bottom, right, (score, row, col, key))
  send(array, dst) / recv(like_shape, src) -> array
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, List, Sequence, Tuple

NO_KEY = (1 << 64) - 1
Best = Tuple[int, int, int, int]  # score, row, col, key


def column_chunks(n: int, world: int, align: int = 256) -> List[Tuple[int, int]]:
    """One column range per rank, as equal as the `align` granularity allows
    (the last chunk takes the remainder); a rank may get an empty range only
    when n is smaller than world * align."""
    if world < 1 or n < 0:
        raise ValueError("bad chunking")
    bounds = [0]
    for g in range(1, world):
        c = int(round(n * g / world / align)) * align
        bounds.append(min(max(c, bounds[-1]), n))
    bounds.append(n)
    return [(bounds[g], bounds[g + 1]) for g in range(world)]


def row_blocks(m: int, height: int) -> List[Tuple[int, int]]:
    """Row blocks of `height` rows (a multiple of 512), the last one shorter."""
    if height <= 0 or height % 512 != 0:
        raise ValueError("block height must be a positive multiple of 512")
    return [(r, min(r + height, m)) for r in range(0, m, height)]


def better(x: Best, y: Best) -> bool:
    """x beats y: higher score, then smaller tie key."""
    return x[0] > y[0] or (x[0] == y[0] and x[0] > 0 and x[3] < y[3])


def merge(cands: Sequence[Best]) -> Best:
    best: Best = (0, 0, 0, NO_KEY)
    for c in cands:
        if c[0] > 0 and better(c, best):
            best = c
    return best


def run_rank(rank: int, world: int, m: int, n: int, height: int, block: Callable, send: Callable,
             recv: Callable) -> Best:
    """The blocks of one rank in order; returns the rank's best cell."""
    chunks = column_chunks(n, world)
    c_lo, c_hi = chunks[rank]
    best: Best = (0, 0, 0, NO_KEY)
    if c_lo == c_hi:
        return best
    # the ranks that own columns form the chain
    prev = max((g for g in range(rank) if chunks[g][0] < chunks[g][1]), default=None)
    nxt = min((g for g in range(rank + 1, world) if chunks[g][0] < chunks[g][1]), default=None)
    top = None
    corner_next = 0  # H[R_b - 1][C_g - 1]: 0 above the first row
    blocks = row_blocks(m, height)
    for b, (r_lo, r_hi) in enumerate(blocks):
        left = None
        corner = 0
        if prev is not None:
            left = recv((r_hi - r_lo, 2), prev)
            corner = corner_next
            corner_next = int(left[-1][0])
        bottom, right, got = block(r_lo, r_hi, c_lo, c_hi, top, left, corner,
                                   b + 1 < len(blocks), nxt is not None)
        if nxt is not None:
            send(right, nxt)
        top = bottom
        if got[0] > 0 and better(got, best):
            best = got
    return best


# ------------------------------------------------------------------ GPU blocks

class GpuBlocks:
    """Block function on the GPU through swb_score_block_device: the pair's
    sequences and the borders live in device memory (torch tensors on this
    rank's GPU); the library runs on the context's stream."""

    def __init__(self, ctx, d_rows, d_cols, sc, flags: int = 0):
        import torch
        from . import lib, SwbError, BlockBest
        self.torch, self.lib, self.SwbError, self.BlockBest = torch, lib(), SwbError, BlockBest
        self.ctx, self.d_rows, self.d_cols, self.sc, self.flags = ctx, d_rows, d_cols, sc, flags
        self.m, self.n = d_rows.numel(), d_cols.numel()
        self.stage1_ms = 0.0

    def __call__(self, r_lo, r_hi, c_lo, c_hi, top, left, corner, want_bottom, want_right):
        torch = self.torch
        dev = self.d_rows.device
        bottom = torch.empty((c_hi - c_lo, 2), dtype=torch.int32, device=dev) if want_bottom else None
        right = torch.empty((r_hi - r_lo, 2), dtype=torch.int32, device=dev) if want_right else None
        out = self.BlockBest()
        ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
        rc = self.lib.swb_score_block_device(
            self.ctx._h, C.c_void_p(self.d_rows.data_ptr() + r_lo), r_hi - r_lo,
            C.c_void_p(self.d_cols.data_ptr() + c_lo), c_hi - c_lo, ptr(top), ptr(left), int(corner), r_lo, c_lo,
            self.m, self.n, C.byref(self.sc), self.flags, ptr(bottom), ptr(right), C.byref(out))
        if rc != 0:
            self.ctx._err(rc)
        self.stage1_ms += out.stage1_ms
        return bottom, right, (out.score, out.row, out.col, out.key)


def torch_links(device=None):
    """send / recv over torch.distributed (NCCL between GPUs, gloo on the CPU):
    recv fills a fresh buffer of the receiver."""
    import torch
    import torch.distributed as dist

    def send(arr, dst):
        dist.send(arr.contiguous(), dst)

    def recv(shape, src):
        buf = torch.empty(shape, dtype=torch.int32, device=device)
        dist.recv(buf, src)
        return buf
    return send, recv


def gather_best(best: Best, device=None) -> Best:
    """Every rank's best cell to every rank (one small all-gather after the
    last block), merged."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size()
    key = best[3]
    mine = torch.tensor([best[0], best[1], best[2], key >> 32, key & 0xFFFFFFFF], dtype=torch.int64, device=device)
    allv = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(allv, mine)
    cands = []
    for t in allv:
        v = [int(x) for x in t.tolist()]
        cands.append((v[0], v[1], v[2], (v[3] << 32) | v[4]))
    return merge(cands)


def run_virtual(world: int, m: int, n: int, height: int, block: Callable) -> Best:
    """All ranks of a chain in one process, rank after rank (rank g only needs
    what ranks < g sent): the same protocol with in-memory links, for one GPU
    or the CPU."""
    boxes = {}

    def make(rank):
        def send(arr, dst):
            boxes.setdefault((rank, dst), []).append(arr)

        def recv(shape, src):
            arr = boxes[(src, rank)].pop(0)
            assert tuple(arr.shape) == tuple(shape), (arr.shape, shape)
            return arr
        return send, recv
    cands = []
    for g in range(world):
        s, r = make(g)
        cands.append(run_rank(g, world, m, n, height, block, s, r))
    return merge(cands)
