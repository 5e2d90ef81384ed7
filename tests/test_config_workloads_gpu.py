"""The exact seeded workloads of the plain small pair and of the 100,000-pair
batch, on the GPU, against the oracle.

* Plain small pair (swb200.synth.plain_small(): 2,000 bp vs 400 + a mutated
  1,200 bp window + 400, scoring 1/-3/-5/-2): score, end cell, the alignment, the
  start cell and every crosspoint equal the oracle's canonical traceback, under
  both tie rules, and the alignment re-scores to the score.
* 100,000-pair batch (swb200.synth.batched(), scoring 2/-3/-5/-2, the best 1%
  traced): the whole batch runs in one call; 2,000 pairs spread over the batch
  get the oracle's score and end cell, and a sample of the traced pairs gets the
  oracle's alignment, start cell and crosspoints.
"""
import numpy as np
import pytest

import oracle_ctypes as O
import swb200
from swb200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tie_flag", [0, swb200.FLAG_TIE_ROWMAJOR])
def test_plain_small_pair_exact_workload(gpu_ctx, tie_flag):
    a, b, sc_t = synth.plain_small()
    assert len(a) == 2000
    rows, cols, swapped = O.orient(a, b)
    sc = O.scoring(*sc_t)
    tie = O.TIE_ROWMAJOR if tie_flag else O.TIE_REFERENCE
    e = O.stage1(rows, cols, sc, O.TEXTBOOK, tie)
    r = gpu_ctx.align(a, b, swb200.scoring(*sc_t), tie_flag)
    assert (r.score, r.end_row, r.end_col, bool(r.swapped)) == (e.score, e.row, e.col, swapped)
    assert e.score > 300  # the mutated window aligns end to end
    ops, sr, scol, xps = O.traceback_xp(rows, cols, sc, e.row, e.col, r.xpoint_interval)
    assert r.ops == ops
    assert (r.start_row, r.start_col) == (sr, scol)
    assert [tuple(x) for x in r.xpoints] == [(sr, scol, 0, 0)] + [tuple(x) for x in xps] + \
        [(e.row, e.col, e.score, 0)]
    assert O.score_ops(rows, cols, sc, sr, scol, r.ops) == e.score


def _oracle_pair(buf, ref, sc):
    q = bytes(buf[ref[0]:ref[0] + ref[1]])
    t = bytes(buf[ref[2]:ref[2] + ref[3]])
    rows, cols, swapped = O.orient(q, t)
    # the AVX-512 wavefront on one thread where the host has it (checked against
    # the scalar oracle in test_oracle.py), else the scalar one
    e = O.stage1_fast(rows, cols, sc, O.TIE_REFERENCE, threads=1)[0]
    return rows, cols, swapped, e


def test_batched_workload_sample_against_the_oracle(gpu_ctx):
    buf, refs, sc_t = synth.batched()
    assert len(refs) == 100_000
    res = gpu_ctx.batch_align(buf, refs, swb200.scoring(*sc_t), trace_frac=0.01)
    assert res.n_traced == 1000
    sc = O.scoring(*sc_t)
    sample = np.linspace(0, len(refs) - 1, 2000).astype(np.int64)
    for i in sample.tolist():
        rows, cols, swapped, e = _oracle_pair(buf, refs[i], sc)
        assert (res.score[i], res.end_row[i], res.end_col[i], bool(res.swapped[i])) == \
            (e.score, e.row, e.col, swapped), i
    # the traced pairs are the 1,000 best scores; check 40 of them in full
    traced = np.flatnonzero(res.traced)
    assert len(traced) == 1000
    assert res.score[traced].min() >= np.sort(res.score)[-1000]
    for i in traced[np.linspace(0, len(traced) - 1, 40).astype(np.int64)].tolist():
        rows, cols, swapped, e = _oracle_pair(buf, refs[i], sc)
        assert (res.score[i], res.end_row[i], res.end_col[i]) == (e.score, e.row, e.col), i
        ops, sr, scol, xps = O.traceback_xp(rows, cols, sc, e.row, e.col, int(res.xpoint_interval[i]))
        assert res.ops[i] == ops, i
        assert (res.start_row[i], res.start_col[i]) == (sr, scol), i
        assert [tuple(x) for x in res.xpoints[i]] == [(sr, scol, 0, 0)] + [tuple(x) for x in xps] + \
            [(e.row, e.col, e.score, 0)], i
