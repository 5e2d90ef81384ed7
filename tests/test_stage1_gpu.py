"""Stage 1 on the GPU (score + end cell) against the oracle and the reference's
goldens, through the C ABI."""
import random

import numpy as np
import pytest

import oracle_ctypes as O
import swb200
from conftest import load_fixture_fasta

pytestmark = pytest.mark.gpu

SCORINGS = [(1, -3, -5, -2), (5, -5, -5, -5), (2, -3, -5, -2), (1, -1, -1, -1), (3, -1, -1, -2)]


@pytest.mark.parametrize("idx", [0, 1, 2, 3, 4])
def test_reference_goldens(gpu_ctx, goldens, idx):
    """Tests/test1.sh .. test5.sh: score and 1-based end cell (test 5: 1.03e13 cells)."""
    g = goldens[idx]
    a, b = load_fixture_fasta(g["a"]), load_fixture_fasta(g["b"])
    r = gpu_ctx.align(a, b, swb200.scoring(*g["scoring"]), swb200.FLAG_SCORE_ONLY)
    assert (r.score, r.end_row + 1, r.end_col + 1) == (g["score"], g["row1"], g["col1"])


def _rand_seq(rng, n, alph):
    return bytes(rng.choice(alph) for _ in range(n))


def _check(ctx, a, b, sc, tie_flag=0):
    r = ctx.align(a, b, swb200.scoring(*sc), swb200.FLAG_SCORE_ONLY | tie_flag)
    rows, cols, swapped = O.orient(a, b)
    tie = O.TIE_ROWMAJOR if tie_flag else O.TIE_REFERENCE
    o = O.stage1(rows, cols, O.scoring(*sc), O.TEXTBOOK, tie)
    assert (r.score, r.end_row, r.end_col, r.swapped) == (o.score, o.row, o.col, swapped), \
        (len(a), len(b), sc, tie_flag)


def test_random_small_pairs_both_tie_rules(gpu_ctx):
    rng = random.Random(101)
    for _ in range(150):
        alph = rng.choice([b"ACGT", b"AC", b"A", b"ACGTN"])
        a = _rand_seq(rng, rng.randint(1, 300), alph)
        b = _rand_seq(rng, rng.randint(1, 300), alph)
        _check(gpu_ctx, a, b, rng.choice(SCORINGS), rng.choice([0, swb200.FLAG_TIE_ROWMAJOR]))


@pytest.mark.parametrize("m", [1, 2, 31, 32, 33, 511, 512, 513, 1023, 1024, 1025, 2048, 4097])
def test_strip_boundaries(gpu_ctx, m):
    rng = random.Random(m)
    a = _rand_seq(rng, m, b"ACGT")
    st = rng.randint(0, max(0, m - 1))
    b = bytearray(a[st:st + max(1, m // 2)])
    for i in range(len(b)):
        if rng.random() < 0.08:
            b[i] = rng.choice(b"ACGT")
    for n_extra in (0, 7):
        bb = bytes(b) + _rand_seq(rng, n_extra, b"ACGT")
        for sc in SCORINGS[:3]:
            _check(gpu_ctx, a, bb, sc)


def test_all_equal_sequences_maximal_ties(gpu_ctx):
    for la, lb in [(100, 100), (100, 37), (777, 777), (1200, 640), (20, 9), (9, 9)]:
        for tie in (0, swb200.FLAG_TIE_ROWMAJOR):
            _check(gpu_ctx, b"A" * la, b"A" * lb, (1, -3, -5, -2), tie)
            _check(gpu_ctx, b"A" * la, b"A" * lb, (5, -5, -5, -5), tie)


def test_byte_identity_any_byte_values(gpu_ctx):
    rng = random.Random(5)
    for _ in range(20):
        a = bytes(rng.randrange(256) for _ in range(rng.randint(50, 400)))
        b = bytes(rng.randrange(256) for _ in range(rng.randint(50, 400)))
        b = b[:20] + a[10:120] + b[20:]
        _check(gpu_ctx, a, b, rng.choice(SCORINGS))


def test_medium_similar_pairs(gpu_ctx):
    rng = random.Random(77)
    for _ in range(6):
        a = _rand_seq(rng, rng.randint(3000, 9000), b"ACGT")
        st = rng.randint(0, len(a) // 2)
        core = bytearray(a[st:st + len(a) // 3])
        for i in range(len(core)):
            if rng.random() < 0.05:
                core[i] = rng.choice(b"ACGT")
        b = _rand_seq(rng, 300, b"ACGT") + bytes(core) + _rand_seq(rng, 500, b"ACGT")
        _check(gpu_ctx, a, b, rng.choice(SCORINGS))


def test_empty_inputs(gpu_ctx):
    r = gpu_ctx.align(b"", b"ACGT", swb200.scoring(1, -3, -5, -2), swb200.FLAG_SCORE_ONLY)
    assert (r.score, r.end_row, r.end_col) == (0, 0, 0)
    r = gpu_ctx.align(b"ACGA", b"TTTT", swb200.scoring(1, -3, -5, -2), swb200.FLAG_SCORE_ONLY)
    assert (r.score, r.end_row, r.end_col) == (0, 0, 0)
    r = gpu_ctx.align(b"ACGT", b"TTTT", swb200.scoring(1, -3, -5, -2), swb200.FLAG_SCORE_ONLY)
    assert (r.score, r.end_row, r.end_col) == (1, 3, 0)


def test_device_pointer_path_matches_host_path(gpu_ctx):
    import torch
    rng = random.Random(9)
    a = _rand_seq(rng, 5000, b"ACGT")
    b = a[1000:3000]
    sc = swb200.scoring(1, -3, -5, -2)
    h = gpu_ctx.align(a, b, sc, swb200.FLAG_SCORE_ONLY)
    ta = torch.frombuffer(bytearray(a), dtype=torch.uint8).cuda()
    tb = torch.frombuffer(bytearray(b), dtype=torch.uint8).cuda()
    d = gpu_ctx.align_device(ta.data_ptr(), len(a), tb.data_ptr(), len(b), sc, swb200.FLAG_SCORE_ONLY)
    assert (h.score, h.end_row, h.end_col) == (d.score, d.end_row, d.end_col)


def test_special_rows_match_oracle():
    rng = random.Random(21)
    a = _rand_seq(rng, 3000, b"ACGT")
    b = a[500:2100]
    sc = (1, -3, -5, -2)
    with swb200.Context(device=0, special_interval=1024) as ctx:
        r = ctx.align(a, b, swb200.scoring(*sc), swb200.FLAG_SCORE_ONLY)
        rows, cols, _ = O.orient(a, b)
        ref = O.special_rows(rows, cols, O.scoring(*sc), 1024)
        assert len(ref) == 2
        for i in range(len(ref)):
            got, interval = ctx.special_row(i, len(cols))
            assert interval == 1024
            np.testing.assert_array_equal(got, ref[i])


def test_bounded_wait_runs_out_and_the_context_stays_usable():
    """A strip whose wait for the strip above runs out ends the launch: the call
    returns SWB_ETIMEOUT (the reference would exit -2, src/SWutils.cpp:19-24) within
    the context's wait limit, every other warp stops at its next wait, and the next
    call on the same context returns the oracle's result.  The stall is made on the
    host side of the kernel's contract: the test flag keeps strip 0 from writing
    its hand-off entries, so nothing ever satisfies strip 1's wait."""
    import time
    rng = random.Random(3)
    a = bytes(rng.choice(b"ACGT") for _ in range(6000))  # 6,000 rows: 12+ strips
    b = bytes(rng.choice(b"ACGT") for _ in range(2500))
    sc_t = (1, -3, -5, -2)
    rows, cols, _ = O.orient(a, b)
    e = O.stage1(rows, cols, O.scoring(*sc_t), O.TEXTBOOK, O.TIE_REFERENCE)
    with swb200.Context(device=0, wait_limit_ms=200) as ctx:
        for flags in (swb200.FLAG_SCORE_ONLY, 0):
            t0 = time.monotonic()
            with pytest.raises(swb200.SwbError) as ei:
                ctx.align(a, b, swb200.scoring(*sc_t), flags | swb200.FLAG_TEST_WITHHOLD)
            assert ei.value.code == swb200.SWB_ETIMEOUT
            assert time.monotonic() - t0 < 10.0
            r = ctx.align(a, b, swb200.scoring(*sc_t), flags)
            assert (r.score, r.end_row, r.end_col) == (e.score, e.row, e.col)
