"""Seeded pairs and the oracle's block function for the chain tests (test
infrastructure: the oracle stands in for swb_score_block_device)."""
import random

import numpy as np

import oracle_ctypes as O


def case(seed):
    """A pair with a long similar region crossing several blocks and chunks."""
    rng = random.Random(seed)
    m = rng.choice([1500, 2100, 3000, 3600])
    a = bytes(rng.choice(b"ACGT") for _ in range(m))
    st = rng.randint(0, m // 4)
    core = bytearray(a[st:st + rng.randint(m // 3, m // 2)])
    for i in range(len(core)):
        if rng.random() < 0.07:
            core[i] = rng.choice(b"ACGT")
    for _ in range(rng.randint(0, 5)):
        p = rng.randrange(len(core))
        if rng.random() < 0.5:
            del core[p:p + rng.randint(1, 5)]
        else:
            core[p:p] = bytes(rng.choice(b"ACGT") for _ in range(rng.randint(1, 5)))
    b = bytes(rng.choice(b"ACGT") for _ in range(rng.randint(0, 400))) + bytes(core)
    rows, cols, _ = O.orient(a, b)
    sc = rng.choice([(1, -3, -5, -2), (2, -3, -5, -2), (5, -5, -5, -5), (1, -1, -1, -1)])
    return rows, cols, sc


def oracle_block(rows, cols, sc_t, tie, as_torch=False):
    sc = O.scoring(*sc_t)
    m, n = len(rows), len(cols)

    def block(r_lo, r_hi, c_lo, c_hi, top, left, corner, want_bottom, want_right):
        t = None if top is None else np.asarray(top)
        lf = None if left is None else np.asarray(left)
        bottom, right, e, key = O.block(rows[r_lo:r_hi], cols[c_lo:c_hi], sc, t, lf, corner, r_lo, c_lo, m, n, tie)
        if as_torch:
            import torch
            bottom, right = torch.from_numpy(bottom), torch.from_numpy(right)
        return (bottom if want_bottom else None), (right if want_right else None), (e.score, e.row, e.col, key)
    return block
