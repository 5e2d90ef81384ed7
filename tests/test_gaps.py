"""Gap lists (swb_gap_lists*, no GPU needed): the alignment as the reference
renderer's per-sequence gap records (src/Visualisation.cpp:11-127).  Rendering
the oracle's alignments from those records with a restatement of visualOutput
gives the same blocks as rendering from the operation string (the CLI's way)."""
import os
import random
import types

import numpy as np
import pytest

import oracle_ctypes as O
import swb200


def _visual_output(first, second, g1, g2, start, end, width=50):
    """visualOutput (src/Visualisation.cpp:49-127) over gap records (begin, length)."""
    off = [start[0], start[1]]
    seqs, gaps, stop = (first, second), (g1, g2), (end[0], end[1])
    in_gap, it = [0, 0], [0, 0]
    blocks = []
    while True:
        lines, done = [], 0
        for s in range(2):
            v = []
            i = 0
            while i < width:
                if in_gap[s]:
                    v.append("-")
                    in_gap[s] -= 1
                elif it[s] < len(gaps[s]) and gaps[s][it[s]][0] == off[s]:
                    in_gap[s] = gaps[s][it[s]][1]
                    it[s] += 1
                    continue
                else:
                    v.append(chr(seqs[s][off[s]]))
                    off[s] += 1
                if off[s] > stop[s]:
                    done += 1
                    break
                i += 1
            lines.append("".join(v))
        mid = "".join("|" if a == b else " " for a, b in zip(lines[0], lines[1]))
        blocks.append((lines[0], mid, lines[1]))
        if done:
            return blocks


def _render_ops(rows, cols, ops, sr, sc, width=50):
    """The CLI's rendering from the operation string (cli.cpp render_alignment)."""
    ri, ci, l0, l2, blocks = sr, sc, [], [], []
    for k, op in enumerate(ops):
        a = b = "-"
        if op == "M":
            a, b = chr(rows[ri]), chr(cols[ci])
            ri += 1
            ci += 1
        elif op == "D":
            a = chr(rows[ri])
            ri += 1
        else:
            b = chr(cols[ci])
            ci += 1
        l0.append(a)
        l2.append(b)
        if len(l0) == width or k + 1 == len(ops):
            blocks.append(("".join(l0), "".join("|" if x == y else " " for x, y in zip(l0, l2)), "".join(l2)))
            l0, l2 = [], []
    return blocks


def _alignment(rng, n, sc):
    a = bytes(rng.choice(b"ACGT") for _ in range(n))
    core = bytearray(a[n // 5: 4 * n // 5])
    for i in range(len(core)):
        if rng.random() < 0.08:
            core[i] = rng.choice(b"ACGT")
    for _ in range(rng.randint(0, 6)):  # indels
        p = rng.randrange(len(core))
        if rng.random() < 0.5:
            del core[p:p + rng.randint(1, 4)]
        else:
            core[p:p] = bytes(rng.choice(b"ACGT") for _ in range(rng.randint(1, 4)))
    b = bytes(rng.choice(b"ACGT") for _ in range(30)) + bytes(core)
    rows, cols, _ = O.orient(a, b)
    e = O.stage1(rows, cols, O.scoring(*sc), O.TEXTBOOK, O.TIE_REFERENCE)
    ops, sr, scol, _ = O.traceback_xp(rows, cols, O.scoring(*sc), e.row, e.col, 20)
    return rows, cols, types.SimpleNamespace(ops=ops, start_row=sr, start_col=scol, end_row=e.row, end_col=e.col)


@pytest.mark.parametrize("seed", range(6))
def test_gap_lists_render_like_the_alignment(seed):
    rng = random.Random(100 + seed)
    sc = (1, -3, -5, -2) if seed % 2 else (2, -3, -5, -2)
    rows, cols, al = _alignment(rng, rng.randint(80, 600), sc)
    assert al.ops and al.ops[0] == "M" and al.ops[-1] == "M"
    g1, g2 = swb200.gap_lists(al)
    assert sum(L for _, L in g1) == al.ops.count("I") and sum(L for _, L in g2) == al.ops.count("D")
    got = _visual_output(rows, cols, g1, g2, (al.start_row, al.start_col), (al.end_row, al.end_col))
    assert got == _render_ops(rows, cols, al.ops, al.start_row, al.start_col)


def test_gap_records_by_hand(tmp_path):
    al = types.SimpleNamespace(ops="MMIIMDDDMM", start_row=5, start_col=7)
    g1, g2 = swb200.gap_lists(al)
    # rows: M M (5, 6) | I I: gap before row 7 | M (7) | D D D (8, 9, 10) | M M (11, 12)
    # cols: M M (7, 8) | I I (9, 10) | M (11) | D D D: gap before col 12 | M M (12, 13)
    assert g1 == [(7, 2)] and g2 == [(12, 3)]
    f1, f2 = os.path.join(tmp_path, "first.bin"), os.path.join(tmp_path, "second.bin")
    swb200.write_gap_lists(al, f1, f2)
    assert np.fromfile(f1, dtype=np.int32).reshape(-1, 2).tolist() == [[7, 2]]
    assert np.fromfile(f2, dtype=np.int32).reshape(-1, 2).tolist() == [[12, 3]]
    assert swb200.gap_lists(types.SimpleNamespace(ops="MMM", start_row=0, start_col=0)) == ([], [])


def test_gap_lists_reject_bad_operations():
    with pytest.raises(swb200.SwbError) as ei:
        swb200.gap_lists(types.SimpleNamespace(ops="MMXM", start_row=0, start_col=0))
    assert ei.value.code == swb200.SWB_EINVAL


def _ops_strategy():
    from hypothesis import strategies as st
    run = st.tuples(st.sampled_from("MID"), st.integers(1, 9))
    return st.lists(run, min_size=0, max_size=30).map(lambda rs: "M" + "".join(o * k for o, k in rs) + "M")


def test_gap_lists_round_trip_property():
    from hypothesis import given, settings
    from hypothesis import strategies as st

    @settings(max_examples=150, deadline=None)
    @given(_ops_strategy(), st.integers(0, 40), st.integers(0, 40), st.integers(0, 2**31 - 1))
    def check(ops, sr, sc, seed):
        rng = random.Random(seed)
        nr, nc = sr + ops.count("M") + ops.count("D") + 5, sc + ops.count("M") + ops.count("I") + 5
        rows = bytes(rng.choice(b"ACGT") for _ in range(nr))
        cols = bytes(rng.choice(b"ACGT") for _ in range(nc))
        er = sr + ops.count("M") + ops.count("D") - 1
        ec = sc + ops.count("M") + ops.count("I") - 1
        al = types.SimpleNamespace(ops=ops, start_row=sr, start_col=sc)
        g1, g2 = swb200.gap_lists(al)
        assert all(L > 0 for _, L in g1 + g2)
        assert [b for b, _ in g1] == sorted(b for b, _ in g1) and [b for b, _ in g2] == sorted(b for b, _ in g2)
        assert _visual_output(rows, cols, g1, g2, (sr, sc), (er, ec)) == _render_ops(rows, cols, ops, sr, sc)

    check()


def _cli_block_text(blocks):
    """The CLI's alignment block as printed (cli.cpp render_alignment)."""
    out = "\n\tVisual representation of the alignment:\n\n"
    for l0, l1, l2 in blocks:
        out += f"\t\t{l0}\n\t\t{l1}\n\t\t{l2}\n\n"
    return out


@pytest.mark.skipif(not os.path.exists(O.VISUAL_PATH), reason="reference renderer not built (make -C oracle ref)")
@pytest.mark.parametrize("seed", range(8))
def test_reference_renderer_prints_the_cli_block(tmp_path, seed):
    """The gap-list files the library writes, rendered by the reference's own
    visualOutput (src/Visualisation.cpp:11-129, CPU build), print exactly the
    block the CLI renders from the operation string, byte for byte."""
    rng = random.Random(300 + seed)
    sc = (1, -3, -5, -2) if seed % 2 else (2, -3, -5, -2)
    rows, cols, al = _alignment(rng, rng.randint(60, 900), sc)
    f1, f2 = os.path.join(tmp_path, "first.gaps"), os.path.join(tmp_path, "second.gaps")
    swb200.write_gap_lists(al, f1, f2)
    got = O.run_reference_visual(rows, cols, f1, f2, (al.start_row, al.start_col), (al.end_row, al.end_col))
    assert got == _cli_block_text(_render_ops(rows, cols, al.ops, al.start_row, al.start_col))


@pytest.mark.skipif(not os.path.exists(O.VISUAL_PATH), reason="reference renderer not built (make -C oracle ref)")
def test_reference_renderer_on_gap_runs_at_block_edges(tmp_path):
    """Gap runs that start, end or straddle the 50-column block boundary, and no gaps at all."""
    rng = random.Random(9)
    for ops in ["M" * 49 + "I" * 3 + "M" * 10, "M" * 50 + "D" * 50 + "M", "M" * 120,
                "M" + "I" * 49 + "M" + "D" * 51 + "M" * 3, "MIMDMIMDM" * 20]:
        sr, scol = rng.randint(0, 9), rng.randint(0, 9)
        rows = bytes(rng.choice(b"ACGT") for _ in range(sr + ops.count("M") + ops.count("D") + 3))
        cols = bytes(rng.choice(b"ACGT") for _ in range(scol + ops.count("M") + ops.count("I") + 3))
        al = types.SimpleNamespace(ops=ops, start_row=sr, start_col=scol)
        er = sr + ops.count("M") + ops.count("D") - 1
        ec = scol + ops.count("M") + ops.count("I") - 1
        f1, f2 = os.path.join(tmp_path, "first.gaps"), os.path.join(tmp_path, "second.gaps")
        swb200.write_gap_lists(al, f1, f2)
        got = O.run_reference_visual(rows, cols, f1, f2, (sr, scol), (er, ec))
        assert got == _cli_block_text(_render_ops(rows, cols, ops, sr, scol)), ops
