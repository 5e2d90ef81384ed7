"""Batched path (swb_batch_align*) on the GPU: every pair of a batch gets
exactly what it gets alone (the oracle and the plain pair path), including the
alignment and crosspoints of the traced pairs."""
import random

import numpy as np
import pytest

import oracle_ctypes as O
import swb200

pytestmark = pytest.mark.gpu


def _pack(pairs):
    buf, refs, off = bytearray(), [], 0
    for a, b in pairs:
        refs.append((off, len(a), off + len(a), len(b)))
        buf += a + b
        off += len(a) + len(b)
    return bytes(buf), np.array(refs, dtype=np.int64).reshape(-1, 4)


def _mutated(rng, n, frac=0.7, sub=0.08, alph=b"ACGT"):
    a = bytes(rng.choice(alph) for _ in range(n))
    st = rng.randint(0, max(0, n - int(n * frac)))
    core = bytearray(a[st:st + int(n * frac)])
    for i in range(len(core)):
        if rng.random() < sub:
            core[i] = rng.choice(alph)
    if core and rng.random() < 0.5:
        del core[rng.randrange(len(core))]
    b = bytes(rng.choice(alph) for _ in range(rng.randint(0, 60))) + bytes(core)
    return (a, b) if rng.random() < 0.5 else (b, a)


def _oracle(a, b, sc, tie):
    rows, cols, swapped = O.orient(a, b)
    if len(cols) == 0:
        return 0, 0, 0, swapped
    o = O.stage1(rows, cols, O.scoring(*sc), O.TEXTBOOK, tie)
    return o.score, o.row, o.col, swapped


@pytest.mark.parametrize("tie_flag", [0, swb200.FLAG_TIE_ROWMAJOR])
def test_random_batch_matches_oracle(gpu_ctx, tie_flag):
    rng = random.Random(7 + tie_flag)
    pairs = []
    for _ in range(240):
        n = rng.choice([1, 3, 17, 200, 511, 512, 513, 900, 1500, 2100])
        pairs.append(_mutated(rng, rng.randint(max(1, n // 2), n)))
    pairs += [(b"", b"ACGT"), (b"ACGT", b""), (b"", b""), (b"A" * 600, b"A" * 300), (b"A" * 40, b"A" * 900)]
    buf, refs = _pack(pairs)
    sc = (2, -3, -5, -2)
    res = gpu_ctx.batch_align(buf, refs, swb200.scoring(*sc), tie_flag)
    tie = O.TIE_ROWMAJOR if tie_flag else O.TIE_REFERENCE
    for i, (a, b) in enumerate(pairs):
        s, r, c, sw = _oracle(a, b, sc, tie)
        assert (res.score[i], res.end_row[i], res.end_col[i], bool(res.swapped[i])) == (s, r, c, sw), i


def test_batch_equals_plain_path_with_traceback(gpu_ctx):
    rng = random.Random(11)
    pairs = [_mutated(rng, rng.randint(300, 3000), frac=0.8) for _ in range(60)]
    pairs.append((b"ACGTACGT" * 10, b"TTTT"))
    buf, refs = _pack(pairs)
    sc = (1, -3, -5, -2)
    res = gpu_ctx.batch_align(buf, refs, swb200.scoring(*sc), 0, trace_frac=0.25)
    assert res.n_traced == 16
    # the traced ones are the 16 best scores (ties: lower index)
    order = sorted(range(len(pairs)), key=lambda i: (-res.score[i], i))[:16]
    assert sorted(order) == [i for i in range(len(pairs)) if res.traced[i]]
    for i, (a, b) in enumerate(pairs):
        p = gpu_ctx.align(a, b, swb200.scoring(*sc), 0 if res.traced[i] else swb200.FLAG_SCORE_ONLY)
        assert (res.score[i], res.end_row[i], res.end_col[i]) == (p.score, p.end_row, p.end_col), i
        if res.traced[i]:
            assert res.ops[i] == p.ops, i
            assert (res.start_row[i], res.start_col[i]) == (p.start_row, p.start_col)
            assert res.xpoints[i] == p.xpoints, i
            assert res.xpoint_interval[i] == p.xpoint_interval


def test_traced_pairs_match_oracle_traceback(gpu_ctx):
    rng = random.Random(12)
    pairs = [_mutated(rng, rng.randint(50, 1200), frac=0.9) for _ in range(40)]
    buf, refs = _pack(pairs)
    sc = (2, -3, -5, -2)
    res = gpu_ctx.batch_align(buf, refs, swb200.scoring(*sc), 0, trace_frac=1.0)
    for i, (a, b) in enumerate(pairs):
        rows, cols, _ = O.orient(a, b)
        e = O.stage1(rows, cols, O.scoring(*sc), O.TEXTBOOK, O.TIE_REFERENCE)
        assert res.score[i] == e.score
        if e.score == 0:
            assert res.ops[i] == "" and res.xpoints[i] == [(e.row, e.col, 0, 0)]
            continue
        ops, sr, scol, xps = O.traceback_xp(rows, cols, O.scoring(*sc), e.row, e.col, int(res.xpoint_interval[i]))
        assert res.ops[i] == ops
        assert (res.start_row[i], res.start_col[i]) == (sr, scol)
        assert res.xpoints[i][1:-1] == xps
        assert O.score_ops(rows, cols, O.scoring(*sc), sr, scol, ops) == e.score


def test_long_pair_inside_a_batch(gpu_ctx):
    """A pair with many strips runs as an intra-sequence wavefront across warps
    while small pairs fill the other warps."""
    rng = random.Random(13)
    big = _mutated(rng, 40_000, frac=0.9, sub=0.05)
    pairs = [_mutated(rng, rng.randint(100, 1500)) for _ in range(500)]
    pairs.insert(123, big)
    buf, refs = _pack(pairs)
    sc = (1, -3, -5, -2)
    res = gpu_ctx.batch_align(buf, refs, swb200.scoring(*sc))
    p = gpu_ctx.align(big[0], big[1], swb200.scoring(*sc), swb200.FLAG_SCORE_ONLY)
    assert (res.score[123], res.end_row[123], res.end_col[123]) == (p.score, p.end_row, p.end_col)
    for i in rng.sample(range(len(pairs)), 40):
        a, b = pairs[i]
        s, r, c, _ = _oracle(a, b, sc, O.TIE_REFERENCE)
        assert (res.score[i], res.end_row[i], res.end_col[i]) == (s, r, c)


def test_any_byte_values_use_the_compare_path(gpu_ctx):
    rng = random.Random(14)
    pairs = []
    for _ in range(50):
        a = bytes(rng.randrange(256) for _ in range(rng.randint(20, 700)))
        b = a[5:300] + bytes(rng.randrange(256) for _ in range(rng.randint(0, 50)))
        pairs.append((a, b))
    buf, refs = _pack(pairs)
    sc = (3, -1, -1, -2)
    res = gpu_ctx.batch_align(buf, refs, swb200.scoring(*sc))
    for i, (a, b) in enumerate(pairs):
        assert (res.score[i], res.end_row[i], res.end_col[i]) == _oracle(a, b, sc, O.TIE_REFERENCE)[:3]


def test_device_buffer_and_repeat_calls(gpu_ctx):
    import torch
    rng = random.Random(15)
    pairs = [_mutated(rng, rng.randint(100, 2000)) for _ in range(100)]
    buf, refs = _pack(pairs)
    sc = swb200.scoring(1, -3, -5, -2)
    d = torch.frombuffer(bytearray(buf), dtype=torch.uint8).cuda()
    r1 = gpu_ctx.batch_align(len(buf), refs, sc, seq_ptr=d.data_ptr(), device=True)
    r2 = gpu_ctx.batch_align(buf, refs, sc)
    assert (r1.score == r2.score).all() and (r1.end_row == r2.end_row).all() and (r1.end_col == r2.end_col).all()


def test_empty_batch_and_bad_ranges(gpu_ctx):
    sc = swb200.scoring(1, -3, -5, -2)
    r = gpu_ctx.batch_align(b"", np.zeros((0, 4), dtype=np.int64), sc)
    assert len(r.score) == 0
    with pytest.raises(swb200.SwbError) as ei:
        gpu_ctx.batch_align(b"ACGT", np.array([[0, 4, 2, 5]], dtype=np.int64), sc)
    assert ei.value.code == swb200.SWB_EINVAL


def _same(r0, r1):
    for f in ("score", "end_row", "end_col", "start_row", "start_col", "swapped", "traced", "xpoint_interval"):
        assert (getattr(r0, f) == getattr(r1, f)).all(), f
    assert r0.ops == r1.ops and r0.xpoints == r1.xpoints and r0.n_traced == r1.n_traced


@pytest.mark.parametrize("trace_frac", [0.0, 0.3, 1.0])
def test_graph_replay_equals_direct_launches(gpu_ctx, monkeypatch, trace_frac):
    """Host batches run as one replayed CUDA graph; the same batch through the
    direct launches gives the same results, and replays reuse the captured graph
    with new sizes in the device header."""
    rng = random.Random(21)
    pairs = [_mutated(rng, rng.randint(40, 2600)) for _ in range(150)]
    pairs += [(b"", b"AC"), (b"A" * 700, b"T" * 600), (b"ACGT" * 300, b"ACGT" * 290)]
    buf, refs = _pack(pairs)
    sc = swb200.scoring(2, -3, -5, -2)
    monkeypatch.setenv("SWB_BATCH_GRAPH", "0")
    r0 = gpu_ctx.batch_align(buf, refs, sc, 0, trace_frac=trace_frac)
    monkeypatch.setenv("SWB_BATCH_GRAPH", "1")
    r1 = gpu_ctx.batch_align(buf, refs, sc, 0, trace_frac=trace_frac)
    _same(r0, r1)
    # a smaller batch, then the first one again: same graph, other sizes
    small = pairs[:7]
    b2, f2 = _pack(small)
    r2 = gpu_ctx.batch_align(b2, f2, sc, 0, trace_frac=trace_frac)
    for i in range(len(small)):
        assert (r2.score[i], r2.end_row[i], r2.end_col[i]) == (r1.score[i], r1.end_row[i], r1.end_col[i])
        if trace_frac == 1.0:
            assert r2.ops[i] == r1.ops[i] and r2.xpoints[i] == r1.xpoints[i]
    _same(r1, gpu_ctx.batch_align(buf, refs, sc, 0, trace_frac=trace_frac))


def test_graph_mode_switch_between_alphabets(gpu_ctx):
    """The table / compare choice is made on the device each replay: a DNA batch,
    a batch with more than four byte values, then DNA again."""
    rng = random.Random(22)
    sc = (1, -3, -5, -2)
    dna = [_mutated(rng, rng.randint(100, 900)) for _ in range(30)]
    prot = [_mutated(rng, rng.randint(100, 900), alph=b"ACDEFGHIKLMNPQRSTVWY") for _ in range(30)]
    for batch in (dna, prot, dna):
        buf, refs = _pack(batch)
        res = gpu_ctx.batch_align(buf, refs, swb200.scoring(*sc), 0, trace_frac=1.0)
        for i, (a, b) in enumerate(batch):
            assert (res.score[i], res.end_row[i], res.end_col[i]) == _oracle(a, b, sc, O.TIE_REFERENCE)[:3], i
            if res.score[i] > 0:
                rows, cols, _ = O.orient(a, b)
                assert O.score_ops(rows, cols, O.scoring(*sc), res.start_row[i], res.start_col[i],
                                   res.ops[i]) == res.score[i]


def _packable_batch(seed, n, extra=()):
    rng = random.Random(seed)
    pairs = []
    for _ in range(n):
        L = rng.choice([40, 300, 600, 1100, 1600, 2400])
        pairs.append(_mutated(rng, rng.randint(max(1, L // 2), L)))
    pairs += list(extra)
    rng.shuffle(pairs)
    return pairs


RL = swb200.FLAG_TIE_ROWMAJOR


@pytest.mark.parametrize("tie_flag,rows_per_lane,whole", [(0, "14", ""), (RL, "14", ""), (0, "8", ""), (RL, "8", ""),
                                                          (0, "14", "64"), (RL, "8", "64"), (0, "14", "0")])
def test_packed_16bit_pass_equals_int32_and_oracle(gpu_ctx, monkeypatch, tie_flag, rows_per_lane, whole):
    """A batch of >= 2,048 pairs in the table mode runs its scoring pass two pairs
    per warp in packed 16-bit lanes (448- or 256-row strips; short pairs strip
    after strip on one warp, long ones chained across warps, or all of them one
    way with SWB_BATCH16_WHOLE); every pair gets exactly the int32 pass's result
    (SWB_BATCH_PACK=0) and, on a sample, the oracle's, under both tie rules; the
    traced pairs' store pass re-checks the packed scores."""
    monkeypatch.setenv("SWB_BATCH16_R", rows_per_lane)
    if whole:
        monkeypatch.setenv("SWB_BATCH16_WHOLE", whole)
    pairs = _packable_batch(21 + tie_flag, 2600, [(b"", b"ACGT"), (b"A" * 600, b"A" * 300)])
    buf, refs = _pack(pairs)
    sc = (2, -3, -5, -2)
    packed = gpu_ctx.batch_align(buf, refs, swb200.scoring(*sc), tie_flag, trace_frac=0.01)
    monkeypatch.setenv("SWB_BATCH_PACK", "0")
    plain = gpu_ctx.batch_align(buf, refs, swb200.scoring(*sc), tie_flag, trace_frac=0.01)
    monkeypatch.delenv("SWB_BATCH_PACK")
    for f in ("score", "end_row", "end_col", "swapped", "start_row", "start_col", "traced"):
        assert np.array_equal(getattr(packed, f), getattr(plain, f)), f
    assert packed.ops == plain.ops
    tie = O.TIE_ROWMAJOR if tie_flag else O.TIE_REFERENCE
    rng = random.Random(3)
    for i in rng.sample(range(len(pairs)), 250):
        a, b = pairs[i]
        s, r, c, sw = _oracle(a, b, sc, tie)
        assert (packed.score[i], packed.end_row[i], packed.end_col[i], bool(packed.swapped[i])) == (s, r, c, sw), i


@pytest.mark.parametrize("rows_per_lane,whole", [("14", ""), ("8", ""), ("14", "64")])
def test_packed_pass_detects_16bit_saturation_and_redoes_in_int32(gpu_ctx, monkeypatch, rows_per_lane, whole):
    """With the test flag every pair is packed, also identical pairs of 17,000 bp
    whose score (2 x 17,000 = 34,000) does not fit 16 bits: the kernel flags
    them when a column maximum reaches the limit and they are scored again in
    int32, so the results equal the int32 pass and the exact answer."""
    monkeypatch.setenv("SWB_BATCH16_R", rows_per_lane)
    if whole:
        monkeypatch.setenv("SWB_BATCH16_WHOLE", whole)
    rng = random.Random(77)
    longs = []
    for L in (17_000, 16_600):
        s = bytes(rng.choice(b"ACGT") for _ in range(L))
        longs.append((s, s))
    pairs = _packable_batch(5, 2100, longs)
    buf, refs = _pack(pairs)
    sc = (2, -3, -5, -2)
    forced = gpu_ctx.batch_align(buf, refs, swb200.scoring(*sc), swb200.FLAG_TEST_PACK_ANY)
    monkeypatch.setenv("SWB_BATCH_PACK", "0")
    plain = gpu_ctx.batch_align(buf, refs, swb200.scoring(*sc))
    monkeypatch.delenv("SWB_BATCH_PACK")
    assert np.array_equal(forced.score, plain.score)
    assert np.array_equal(forced.end_row, plain.end_row) and np.array_equal(forced.end_col, plain.end_col)
    for s, _ in longs:
        i = next(k for k, p in enumerate(pairs) if p[0] == s and p[1] == s)
        assert (forced.score[i], forced.end_row[i], forced.end_col[i]) == (2 * len(s), len(s) - 1, len(s) - 1)
