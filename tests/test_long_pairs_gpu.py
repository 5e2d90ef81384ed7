"""The full-size pairs on the GPU.  The 1 Mbp pair's score and end cell are
pinned by the oracle's full CPU wavefront (tests/golden/long_pair_golden.json,
made by tests/golden/make_long_pair_golden.py, both tie rules); its alignment and
the 10 Mbp pair's (whose score and end cell the oracle's AVX-512 wavefront pins,
tests/golden/chromosome_golden.json) are checked through properties that hold at any size: the
operations re-score to the reported score from a start cell to the end cell, the
crosspoints lie on the path with its prefix score on every special row, and
stage 1 gives the same result with another tile height."""
import hashlib
import json
import os

import numpy as np
import pytest

import swb200
from conftest import GOLDEN
from swb200 import synth

pytestmark = pytest.mark.gpu


def _path_check(rows: bytes, cols: bytes, sc, res):
    """Scores the path of res.ops from its start cell; returns the checks' data."""
    match, mismatch, open_, ext = sc
    o = np.frombuffer(res.ops.encode(), np.uint8)
    assert o.size > 0 and o[0] == ord("M") and o[-1] == ord("M")
    isM, isI, isD = o == ord("M"), o == ord("I"), o == ord("D")
    assert (isM | isI | isD).all()
    dr, dc = (isM | isD).astype(np.int64), (isM | isI).astype(np.int64)
    cr = res.start_row + np.cumsum(dr) - 1  # cell after each operation
    cc = res.start_col + np.cumsum(dc) - 1
    R, Cs = np.frombuffer(rows, np.uint8), np.frombuffer(cols, np.uint8)
    s = np.zeros(o.size, np.int64)
    mi = np.flatnonzero(isM)
    s[mi] = np.where(R[cr[mi]] == Cs[cc[mi]], match, mismatch)
    prev = np.concatenate([[0], o[:-1]])
    g = isI | isD
    s[g] = np.where(prev[g] == o[g], ext, open_)
    cum = np.cumsum(s)
    assert (cr[-1], cc[-1]) == (res.end_row, res.end_col)
    assert cum[-1] == res.score
    assert cum.min() > 0  # a local alignment never passes through a cell of score <= 0
    # crosspoints: [start (score 0), every special row the path leaves downwards, end]
    X = res.xpoint_interval
    xps = res.xpoints
    assert xps[0] == (res.start_row, res.start_col, 0, 0)
    assert xps[-1] == (res.end_row, res.end_col, res.score, 0)
    want = [r for r in range(((res.start_row + 1 + X - 1) // X) * X - 1, res.end_row, X) if r >= res.start_row]
    assert [x[0] for x in xps[1:-1]] == want
    for (xr, xc, xs, xg) in xps[1:-1]:
        k = int(np.searchsorted(cr, xr, side="right")) - 1  # last cell of the path on row xr
        assert (cr[k], cc[k]) == (xr, xc)
        assert cum[k] == xs
        assert xg in (0, 1) and (xg == 0 or o[k + 1] == ord("D"))
    return cum


def test_long_pair_1mbp_against_the_oracle_golden():
    path = os.path.join(GOLDEN, "long_pair_golden.json")
    gold = json.load(open(path))
    a, b, sc = synth.long_pair()
    assert hashlib.sha256(a).hexdigest() == gold["sha256_a"] and hashlib.sha256(b).hexdigest() == gold["sha256_b"]
    ctx = swb200.Context(device=0)
    try:
        res = ctx.align(a, b, swb200.scoring(*sc))
        g = gold["reference"]
        assert (res.score, res.end_row, res.end_col) == (g["score"], g["end_row"], g["end_col"])
        rows, cols = (b, a) if res.swapped else (a, b)
        _path_check(rows, cols, sc, res)
        r2 = ctx.align(a, b, swb200.scoring(*sc), swb200.FLAG_SCORE_ONLY | swb200.FLAG_TIE_ROWMAJOR)
        g = gold["rowmajor"]
        assert (r2.score, r2.end_row, r2.end_col) == (g["score"], g["end_row"], g["end_col"])
    finally:
        ctx.close()


def test_chromosome_pair_10mbp_properties():
    a, b, sc = synth.chromosome_pair()
    ctx = swb200.Context(device=0, hbm_budget_bytes=40 * 10**9)
    try:
        res = ctx.align(a, b, swb200.scoring(*sc))
        rows, cols = (b, a) if res.swapped else (a, b)
        _path_check(rows, cols, sc, res)
        # the oracle's full-matrix result (AVX-512 wavefront over all 10^14 cells)
        gpath = os.path.join(GOLDEN, "chromosome_golden.json")
        if os.path.exists(gpath):
            g = json.load(open(gpath))
            assert g["sha256_a"] == hashlib.sha256(a).hexdigest() and g["sha256_b"] == hashlib.sha256(b).hexdigest()
            assert (res.score, res.end_row, res.end_col) == \
                (g["reference"]["score"], g["reference"]["end_row"], g["reference"]["end_col"])
        # stage 1 alone, with the other tile height, gives the same score and end cell
        os.environ["SWB_STAGE1_R"] = "8"
        try:
            r8 = ctx.align(a, b, swb200.scoring(*sc), swb200.FLAG_SCORE_ONLY)
        finally:
            os.environ.pop("SWB_STAGE1_R", None)
        assert (r8.score, r8.end_row, r8.end_col) == (res.score, res.end_row, res.end_col)
    finally:
        ctx.close()
