"""How a crosspoint list printed by the reference's own stage 2 relates to the
oracle's canonical traceback (test infrastructure: used by
tests/golden/make_fixtures.py to label refemu_stage2.json and by the tests that
re-check those labels and compare the GPU with the reference's lists).

The reference prints [start (score 0), crosspoints top to bottom, end]
(src/main.cu:243-248, list built by src/Crosspointer.cpp:104-108, crosspoints
joined by getTracebackScore, src/SWutils.cpp:175-231, start by findStartX,
src/Crosspointer.cpp:263-318).  All coordinates are 0-based.
"""
from __future__ import annotations

import oracle_ctypes as O


def on_optimal_path(rows: bytes, cols: bytes, s, x, er: int, ec: int, best: int) -> bool:
    """Crosspoint x = (row, col, score, gap=0) lies on an optimal alignment ending at
    (er, ec): the forward H there is `score`, and the best continuation from it to
    the end cell adds exactly best - score."""
    r, c, v, gap = x
    if gap != 0 or r > er or c > ec:
        return False
    h = int(O.special_rows(rows[:r + 1], cols, s, r + 1)[0][c][0])
    sub = s.match if rows[r] == cols[c] else s.mismatch
    return h == v and O.anchored_score(rows, cols, s, r, c, er, ec) - sub + v == best


def relation(a: bytes, b: bytes, sc, ref):
    """How the reference's list relates to the oracle's canonical traceback
    [start (score 0), crosspoints top to bottom, end]:
      equal                the same list
      crosspoints_missed   same start and end, the reference's crosspoints are a
                           subset of the canonical ones (its window search missed some)
      other_path           same start and end, some reference crosspoint lies on
                           another optimal path (equal scores)
      other_optimal_start  the reference's start differs and begins another optimal
                           alignment ending at the same end cell
      start_not_found      the list has no start entry (the reference's start
                           search found nothing); its crosspoints lie on optimal paths
      shipped_carry_end    the reference's stage 1 ended elsewhere because of its
                           left-boundary carry (the oracle's ORC_SHIPPED_CARRY mode)
    Every class but the last asserts that each reference crosspoint lies on an
    optimal alignment to the same end cell."""
    rows, cols, _ = O.orient(a, b)
    s = O.scoring(*sc)
    e = O.stage1(rows, cols, s, O.TEXTBOOK, O.TIE_REFERENCE)
    interval = 4 * O.geometry(len(rows), len(cols)).T
    ops, sr, scol, xps = O.traceback_xp(rows, cols, s, e.row, e.col, interval)
    ours = [(sr, scol, 0, 0)] + [tuple(x) for x in xps] + [(e.row, e.col, e.score, 0)]
    ref = [tuple(x) for x in ref]
    if ref == ours:
        return "equal"
    if ref[-1] != ours[-1]:
        c = O.stage1(rows, cols, s, O.SHIPPED_CARRY, O.TIE_REFERENCE)
        assert ref[-1][:3] == (c.row, c.col, c.score), (ref, c)
        return "shipped_carry_end"
    has_start = ref[0][2] == 0
    xs = ref[1:-1] if has_start else ref[:-1]
    assert all(on_optimal_path(rows, cols, s, x, e.row, e.col, e.score) for x in xs), (ref, ours)
    if not has_start:
        return "start_not_found"
    assert O.anchored_score(rows, cols, s, ref[0][0], ref[0][1], e.row, e.col) == e.score, (ref, ours)
    if ref[0] != ours[0]:
        return "other_optimal_start"
    return "crosspoints_missed" if all(x in ours for x in xs) else "other_path"
