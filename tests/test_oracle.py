"""The CPU oracle, pinned before it is trusted.

1. Textbook mode against the goldens the reference ships (Tests/test1-3.sh here;
   test 4 is 1.1e12 cells and runs in the GPU suite against the same golden).
2. Shipped-carry mode against the reference's own kernels compiled for the CPU
   (oracle/refemu), recorded in tests/golden/refemu_cases.json.
3. Internal consistency: multithreaded == single-thread, traceback score ==
   best score, traceback against an independent brute-force recursion.
"""
import random

import pytest

import oracle_ctypes as O
from conftest import load_fixture_fasta, load_json


@pytest.mark.parametrize("idx", [0, 1])
def test_textbook_goldens_small(goldens, idx):
    g = goldens[idx]
    a, b = load_fixture_fasta(g["a"]), load_fixture_fasta(g["b"])
    rows, cols, _ = O.orient(a, b)
    r = O.stage1(rows, cols, O.scoring(*g["scoring"]), O.TEXTBOOK, O.TIE_REFERENCE)
    assert (r.score, r.row + 1, r.col + 1) == (g["score"], g["row1"], g["col1"])


def test_textbook_golden_test3_multithreaded(goldens):
    g = goldens[2]
    a, b = load_fixture_fasta(g["a"]), load_fixture_fasta(g["b"])
    rows, cols, _ = O.orient(a, b)
    r, _ = O.stage1_mt(rows, cols, O.scoring(*g["scoring"]))
    assert (r.score, r.row + 1, r.col + 1) == (g["score"], g["row1"], g["col1"])


def test_shipped_carry_matches_reference_build():
    cases = load_json("refemu_cases.json")
    assert len(cases) >= 200
    bad = []
    for c in cases:
        a, b = c["a"].encode(), c["b"].encode()
        rows, cols, _ = O.orient(a, b)
        g = O.geometry(len(rows), len(cols))
        assert (g.G, g.T, g.P1, g.P2) == (c["G"], c["T"], c["P1"], c["P2"])
        r = O.stage1(rows, cols, O.scoring(*c["scoring"]), O.SHIPPED_CARRY, O.TIE_REFERENCE)
        if (r.score, r.row + 1, r.col + 1) != (c["score"], c["row1"], c["col1"]):
            bad.append((c, r))
    assert not bad, bad[:3]


def test_reference_build_on_real_fixtures():
    """The shipped reference disagrees with its own test-1 golden (carry), agrees
    on test 2, and its stage 2 either hangs or yields only trivial lists."""
    runs = load_json("refemu_fixtures.json")
    for run in runs:
        a, b = load_fixture_fasta(run["a"]), load_fixture_fasta(run["b"])
        rows, cols, _ = O.orient(a, b)
        carry = O.stage1(rows, cols, O.scoring(*run["scoring"]), O.SHIPPED_CARRY)
        assert (carry.score, carry.row + 1, carry.col + 1) == (run["score"], run["row1"], run["col1"])
    assert runs[0]["score"] == 520  # golden says 480: the carry lifts the path start
    assert "timeout_s" in runs[1]["stage2"]


def _rand_pair(rng, lo=1, hi=300):
    alph = rng.choice([b"ACGT", b"AC", b"A", b"ACGTN"])
    a = bytes(rng.choice(alph) for _ in range(rng.randint(lo, hi)))
    b = bytes(rng.choice(alph) for _ in range(rng.randint(lo, hi)))
    return a, b


def test_multithreaded_equals_single_thread():
    rng = random.Random(7)
    for _ in range(120):
        a, b = _rand_pair(rng, 1, 500)
        rows, cols, _ = O.orient(a, b)
        sc = O.scoring(*rng.choice([(1, -3, -5, -2), (5, -5, -5, -5), (2, -3, -5, -2)]))
        for tie in (O.TIE_REFERENCE, O.TIE_ROWMAJOR):
            x = O.stage1(rows, cols, sc, O.TEXTBOOK, tie)
            y, _ = O.stage1_mt(rows, cols, sc, tie, threads=rng.randint(1, 8))
            assert (x.score, x.row, x.col) == (y.score, y.row, y.col)


def _gap_cost(x, y, sc):
    """Best cost of x column-gap and y row-gap characters placed between two
    aligned pairs, split into k runs (each run pays gap_open once, every other
    character gap_extend).  The recurrence lets a run restart through H, so any
    k from the fewest possible runs to x + y is reachable."""
    if x == 0 and y == 0:
        return 0
    kmin = 1 if (x == 0 or y == 0) else 2
    return max(k * sc.gap_open + (x + y - k) * sc.gap_extend for k in range(kmin, x + y + 1))


def _brute_best(rows, cols, sc):
    """Independent check: best local score by enumerating the previous aligned
    pair of every aligned pair (explicit gap blocks, no E/F recurrence)."""
    m, n = len(rows), len(cols)
    best = {}
    top = 0
    for i in range(m):
        for j in range(n):
            s = sc.match if rows[i] == cols[j] else sc.mismatch
            prev = 0
            for i2 in range(i):
                for j2 in range(j):
                    prev = max(prev, best[(i2, j2)] + _gap_cost(j - j2 - 1, i - i2 - 1, sc))
            best[(i, j)] = s + prev
            top = max(top, best[(i, j)])
    return top


def test_textbook_against_brute_force():
    rng = random.Random(11)
    for _ in range(150):
        a, b = _rand_pair(rng, 1, 9)
        rows, cols, _ = O.orient(a, b)
        sc = O.scoring(*rng.choice([(1, -3, -5, -2), (5, -5, -5, -5), (2, -1, -3, -1), (3, -1, -1, -2)]))
        assert O.stage1(rows, cols, sc, O.TEXTBOOK).score == _brute_best(rows, cols, sc)


def test_traceback_scores_and_bounds():
    rng = random.Random(13)
    for _ in range(200):
        a, b = _rand_pair(rng, 1, 200)
        rows, cols, _ = O.orient(a, b)
        sc = O.scoring(*rng.choice([(1, -3, -5, -2), (5, -5, -5, -5), (2, -3, -5, -2), (1, -1, -1, -1)]))
        r = O.stage1(rows, cols, sc, O.TEXTBOOK)
        if r.score == 0:
            continue
        ops, sr, sc_ = O.traceback(rows, cols, sc, r.row, r.col)
        assert ops[0] == "M" and ops[-1] == "M"
        assert O.score_ops(rows, cols, sc, sr, sc_, ops) == r.score
        assert sr + ops.count("M") + ops.count("D") - 1 == r.row
        assert sc_ + ops.count("M") + ops.count("I") - 1 == r.col


def _simd_available():
    return O.stage1_simd(b"ACGT", b"ACG", O.scoring(1, -3, -5, -2), threads=1) is not None


@pytest.mark.skipif(not _simd_available(), reason="CPU without AVX-512")
def test_simd_wavefront_equals_scalar_oracle():
    """orc_stage1_simd (16-row strips, one row per lane, blocks handed between
    threads) gives the scalar oracle's score and end cell under both tie rules,
    on ragged sizes around the strip height and the column block width."""
    rng = random.Random(31)
    for _ in range(160):
        alph = rng.choice([b"ACGT", b"AC", b"A", b"ACGTN"])
        m = rng.choice([1, 2, 15, 16, 17, 33, 100, 1000, 4097])
        n = rng.choice([1, 3, 14, 15, 16, 17, 300, 4095, 4097, 8200])
        a = bytes(rng.choice(alph) for _ in range(m))
        if rng.random() < 0.5 and n <= m:
            st = rng.randint(0, m - n)
            b = bytes(c if rng.random() > 0.1 else rng.choice(alph) for c in a[st:st + n])
        else:
            b = bytes(rng.choice(alph) for _ in range(n))
        rows, cols, _ = O.orient(a, b)
        sc = O.scoring(*rng.choice([(1, -3, -5, -2), (5, -5, -5, -5), (2, -3, -5, -2), (1, -1, -1, -1)]))
        (r0, r1), _ = O.stage1_simd_both(rows, cols, sc, threads=rng.choice([1, 2, 5, 8]))
        e0 = O.stage1(rows, cols, sc, O.TEXTBOOK, O.TIE_REFERENCE)
        e1 = O.stage1(rows, cols, sc, O.TEXTBOOK, O.TIE_ROWMAJOR)
        assert (r0.score, r0.row, r0.col) == (e0.score, e0.row, e0.col), (m, n)
        assert (r1.score, r1.row, r1.col) == (e1.score, e1.row, e1.col), (m, n)


@pytest.mark.skipif(not _simd_available(), reason="CPU without AVX-512")
def test_simd_wavefront_on_test3_golden(goldens):
    """The reference's Tests/test3.sh golden (2.8e10 cells) through the AVX-512 wavefront."""
    g = goldens[2]
    a, b = load_fixture_fasta(g["a"]), load_fixture_fasta(g["b"])
    rows, cols, _ = O.orient(a, b)
    r, _ = O.stage1_simd(rows, cols, O.scoring(*g["scoring"]))
    assert (r.score, r.row + 1, r.col + 1) == (g["score"], g["row1"], g["col1"])


def test_anchored_score_from_the_canonical_start():
    """An alignment from the canonical traceback's start cell to the end cell
    scores exactly the best score; one cell to the right of the start it can
    only score less or the same."""
    rng = random.Random(5)
    for _ in range(40):
        a = bytes(rng.choice(b"ACGT") for _ in range(rng.randint(20, 150)))
        b = bytes(c if rng.random() > 0.1 else rng.choice(b"ACGT") for c in a[5:rng.randint(20, len(a))])
        rows, cols, _ = O.orient(a, b)
        sc = O.scoring(*rng.choice([(1, -3, -5, -2), (5, -5, -5, -5), (1, -1, -1, -1)]))
        e = O.stage1(rows, cols, sc)
        if e.score == 0:
            continue
        ops, sr, scol = O.traceback(rows, cols, sc, e.row, e.col)
        assert O.anchored_score(rows, cols, sc, sr, scol, e.row, e.col) == e.score
        if scol + 1 <= e.col:
            assert O.anchored_score(rows, cols, sc, sr, scol + 1, e.row, e.col) <= e.score
    assert O.anchored_score(b"AC", b"AC", sc, 1, 1, 0, 0) == -(2 ** 63)
