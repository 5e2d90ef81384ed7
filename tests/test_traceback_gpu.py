"""Stage 2 on the GPU (alignment ops, start cell, crosspoints) against the
oracle's full-matrix traceback with the same precedence, through the C ABI."""
import os
import random
import subprocess

import pytest

import oracle_ctypes as O
import swb200
from conftest import GOLDEN, load_fixture_fasta

pytestmark = pytest.mark.gpu

SCORINGS = [(1, -3, -5, -2), (5, -5, -5, -5), (2, -3, -5, -2), (1, -1, -1, -1), (3, -1, -1, -2), (2, -1, -1, -3)]


def _expected(a, b, sc_t, interval):
    rows, cols, swapped = O.orient(a, b)
    sc = O.scoring(*sc_t)
    e = O.stage1(rows, cols, sc, O.TEXTBOOK, O.TIE_REFERENCE)
    if e.score == 0:
        return e, "", e.row, e.col, []
    ops, sr, scol, xps = O.traceback_xp(rows, cols, sc, e.row, e.col, interval)
    return e, ops, sr, scol, xps


def _check(ctx, a, b, sc_t):
    r = ctx.align(a, b, swb200.scoring(*sc_t))
    e, ops, sr, scol, xps = _expected(a, b, sc_t, r.xpoint_interval)
    assert (r.score, r.end_row, r.end_col) == (e.score, e.row, e.col)
    if e.score == 0:
        assert r.ops == ""
        return r
    assert r.ops == ops, (len(a), len(b), sc_t)
    assert (r.start_row, r.start_col) == (sr, scol)
    # [start, crosspoints top -> bottom, end]
    assert r.xpoints[0] == (sr, scol, 0, 0)
    assert r.xpoints[-1] == (e.row, e.col, e.score, 0)
    assert [(x[0], x[1], x[2], x[3]) for x in r.xpoints[1:-1]] == xps
    return r


def _similar_pair(rng, m, frac, sub=0.08, indel=0.02):
    a = bytes(rng.choice(b"ACGT") for _ in range(m))
    st = rng.randint(0, max(0, m - int(m * frac)))
    out = bytearray()
    for ch in a[st:st + int(m * frac)]:
        x = rng.random()
        if x < indel / 2:
            continue
        if x < indel:
            out += bytes(rng.choice(b"ACGT") for _ in range(rng.randint(1, 6)))
        out.append(rng.choice(b"ACGT") if rng.random() < sub else ch)
    b = bytes(rng.choice(b"ACGT") for _ in range(rng.randint(0, 300))) + bytes(out) + \
        bytes(rng.choice(b"ACGT") for _ in range(rng.randint(0, 300)))
    return a, b


def test_random_pairs_match_oracle(gpu_ctx):
    rng = random.Random(404)
    for _ in range(60):
        alph = rng.choice([b"ACGT", b"AC", b"A"])
        a = bytes(rng.choice(alph) for _ in range(rng.randint(1, 700)))
        b = bytes(rng.choice(alph) for _ in range(rng.randint(1, 700)))
        _check(gpu_ctx, a, b, rng.choice(SCORINGS))


def test_similar_pairs_cross_many_blocks(gpu_ctx):
    rng = random.Random(505)
    for m in (1500, 3000, 5200):
        a, b = _similar_pair(rng, m, 0.8)
        for sc_t in SCORINGS[:3] + SCORINGS[4:]:
            _check(gpu_ctx, a, b, sc_t)


def test_level1_mode_matches_oracle():
    """A tiny HBM budget forces the coarse store grid: level-1 cells are
    recomputed by the stage-1 kernel on the GPU before the walk."""
    rng = random.Random(606)
    with swb200.Context(device=0, hbm_budget_bytes=1 << 20) as ctx:
        for m in (2600, 6000):
            a, b = _similar_pair(rng, m, 0.85)
            r = _check(ctx, a, b, (1, -3, -5, -2))
            assert r.kernel_launches > 4


def _shifted_pair(rng, m, cut_lo, cut_len, ins_len, sub=0.03):
    """B = A with a deletion of cut_len bases at cut_lo and an insertion of ins_len
    random bases further on: the alignment runs off the main diagonal, so the
    walker's predicted corridors miss and it has to predict again."""
    a = bytes(rng.choice(b"ACGT") for _ in range(m))
    core = bytearray(a[:cut_lo] + a[cut_lo + cut_len:])
    for i in range(len(core)):
        if rng.random() < sub:
            core[i] = rng.choice(b"ACGT")
    at = len(core) * 3 // 4
    core[at:at] = bytes(rng.choice(b"ACGT") for _ in range(ins_len))
    return a, bytes(core)


def test_path_far_off_the_diagonal(gpu_ctx):
    rng = random.Random(707)
    for m, cut_lo, cut_len, ins_len in [(12000, 3000, 2500, 1800), (9000, 500, 4000, 300)]:
        a, b = _shifted_pair(rng, m, cut_lo, cut_len, ins_len)
        _check(gpu_ctx, a, b, (1, -3, -5, -2))
        _check(gpu_ctx, a, b, (2, -3, -5, -2))


def test_level1_corridor_off_the_diagonal():
    """Level-1 cells (coarse grid forced by a small budget) along a path with
    long gaps: several corridor rounds of level-1 recomputes."""
    rng = random.Random(808)
    with swb200.Context(device=0, hbm_budget_bytes=2 << 20) as ctx:
        a, b = _shifted_pair(rng, 16000, 4000, 3000, 1500)
        _check(ctx, a, b, (1, -3, -5, -2))
        a, b = _similar_pair(rng, 14000, 0.9)
        _check(ctx, a, b, (2, -3, -5, -2))


def test_reference_fixtures(gpu_ctx):
    for fa, fb, sc_t in [("1/A00142.fna.gz", "1/A00145.fna.gz", (5, -5, -5, -5)),
                         ("2/NC_005046.fna.gz", "2/NC_012557.fna.gz", (5, -5, -5, -5)),
                         ("0/seq0.fna.gz", "0/seq1.fna.gz", (5, -5, -5, -5)),
                         ("0/seq5.fna.gz", "0/seq6.fna.gz", (1, -3, -5, -2)),
                         ("0/seq3.fna.gz", "0/seq4.fna.gz", (1, -3, -5, -2))]:
        _check(gpu_ctx, load_fixture_fasta(fa), load_fixture_fasta(fb), sc_t)


def test_long_alignment_is_optimal(gpu_ctx):
    """100 kbp similar pair: the GPU alignment scores exactly the best score and
    spans start..end (size-independent properties; no full-matrix oracle)."""
    rng = random.Random(707)
    a, b = _similar_pair(rng, 100_000, 0.9, sub=0.05, indel=0.01)
    sc_t = (1, -3, -5, -2)
    r = gpu_ctx.align(a, b, swb200.scoring(*sc_t))
    rows, cols, _ = O.orient(a, b)
    assert O.score_ops(rows, cols, O.scoring(*sc_t), r.start_row, r.start_col, r.ops) == r.score
    assert r.start_row + r.ops.count("M") + r.ops.count("D") - 1 == r.end_row
    assert r.start_col + r.ops.count("M") + r.ops.count("I") - 1 == r.end_col
    assert r.score > 50_000


def test_cli_prints_reference_lines(tmp_path):
    fa = tmp_path / "a.fna"
    fb = tmp_path / "b.fna"
    import gzip
    fa.write_bytes(gzip.open(os.path.join(GOLDEN, "seqs", "1", "A00142.fna.gz")).read())
    fb.write_bytes(gzip.open(os.path.join(GOLDEN, "seqs", "1", "A00145.fna.gz")).read())
    p = subprocess.run([swb200.CLI_PATH, str(fa), str(fb), "5", "-5", "-5", "-5"], capture_output=True, text=True)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "\t>Alignment score: 480 at [623, 561]\n\n" in p.stdout
    assert "\t>Cell updates per second: " in p.stdout
    assert "Found " in p.stdout and "\t>xPoint[0]: [" in p.stdout
    assert "Visual representation of the alignment" in p.stdout


def test_448_row_blocks(gpu_ctx, monkeypatch):
    """Stage 1 with 448-row strips (14 rows per lane): special rows every 448 rows
    and the walker's block grid at that spacing give the oracle's alignment."""
    monkeypatch.setenv("SWB_STAGE1_R", "14")
    rng = random.Random(31)
    for m in (700, 2300, 5100):
        a, b = _similar_pair(rng, m, 0.85)
        r = _check(gpu_ctx, a, b, (1, -3, -5, -2))
        assert r.special_interval == 448
    # more than four byte values: the compare path of the same kernels
    a, b = _similar_pair(rng, 3000, 0.85)
    a = a.replace(b"A", b"N", 40)
    r = _check(gpu_ctx, a, b, (2, -3, -5, -2))
    assert r.special_interval == 448


@pytest.mark.skipif(not os.path.exists(O.VISUAL_PATH), reason="reference renderer not built (make -C oracle ref)")
@pytest.mark.parametrize("fixture", [("1/A00142.fna.gz", "1/A00145.fna.gz", ("5", "-5", "-5", "-5")),
                                     ("0/seq3.fna.gz", "0/seq4.fna.gz", ("1", "-3", "-5", "-2"))])
def test_cli_block_equals_the_reference_renderer(tmp_path, fixture):
    """The SWalign CLI's alignment block, and the reference's own visualOutput
    (src/Visualisation.cpp:11-129, CPU build) run on the gap-list files the same
    CLI run wrote (SWB_GAP_LISTS), are the same text byte for byte."""
    import gzip
    fa, fb, sc = fixture
    pa, pb = tmp_path / "a.fna", tmp_path / "b.fna"
    pa.write_bytes(gzip.open(os.path.join(GOLDEN, "seqs", fa)).read())
    pb.write_bytes(gzip.open(os.path.join(GOLDEN, "seqs", fb)).read())
    prefix = str(tmp_path / "gaps")
    env = dict(os.environ, SWB_GAP_LISTS=prefix)
    p = subprocess.run([swb200.CLI_PATH, str(pa), str(pb), *sc], capture_output=True, text=True, env=env)
    assert p.returncode == 0, p.stdout + p.stderr
    out = p.stdout
    k = out.index("\n\tVisual representation of the alignment:\n\n")
    block = out[k:]
    xps = [line for line in out.splitlines() if line.startswith("\t>xPoint[")]
    start = tuple(int(v) for v in xps[0].split("[")[2].split("]")[0].split(","))
    end = tuple(int(v) for v in xps[-1].split("[")[2].split("]")[0].split(","))
    rows, cols, _ = O.orient(load_fixture_fasta(fa), load_fixture_fasta(fb))
    ref = O.run_reference_visual(rows, cols, prefix + ".first.bin", prefix + ".second.bin", start, end)
    assert block == ref


def test_special_rows_and_columns_spilled_to_pinned_host_memory():
    """Stores over the HBM budget but within budget + host_spill_bytes stay on the
    direct grid with the special rows, the special columns or both in mapped
    pinned host memory (the reference appends its special rows to disk files,
    src/Builders.cpp:41-61): the same alignment, start and crosspoints as with
    everything in HBM, and the oracle's score and end cell."""
    rng = random.Random(12)
    a, b = _similar_pair(rng, 60_000, 0.7, sub=0.05, indel=0.01)
    sc = swb200.scoring(1, -3, -5, -2)
    with swb200.Context(device=0) as ctx:
        full = ctx.align(a, b, sc)
    assert full.host_bytes == 0 and full.special_interval in (448, 512)
    rows_b = 8 * (max(len(a), len(b)) // full.special_interval) * min(len(a), len(b))
    cols_b = 8 * (min(len(a), len(b)) // 256) * max(len(a), len(b))
    for budget, spill, expect in [(cols_b + 1024, rows_b + (1 << 20), rows_b),   # rows to the host
                                  (rows_b + 1024, cols_b + (1 << 20), cols_b),   # columns to the host
                                  (1 << 20, rows_b + cols_b + (1 << 21), rows_b + cols_b)]:
        with swb200.Context(device=0, hbm_budget_bytes=budget, host_spill_bytes=spill) as ctx:
            r = ctx.align(a, b, sc)
        assert r.special_interval == full.special_interval  # the direct grid, not level 1
        assert r.host_bytes == expect, (budget, spill, r.host_bytes)
        assert (r.score, r.end_row, r.end_col, r.start_row, r.start_col) == \
            (full.score, full.end_row, full.end_col, full.start_row, full.start_col)
        assert r.ops == full.ops and r.xpoints == full.xpoints
    rows, cols, _ = O.orient(a, b)
    e = O.stage1_fast(rows, cols, O.scoring(1, -3, -5, -2), O.TIE_REFERENCE)[0]
    assert (full.score, full.end_row, full.end_col) == (e.score, e.row, e.col)
