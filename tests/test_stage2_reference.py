"""Stage 2 (start cell, crosspoints) against the reference's OWN stage 2.

The reference's crosspoint lists come from its sources compiled for the CPU
(oracle/_ref/swalign_emu, the committed recipe in oracle/Makefile), run by
tests/golden/make_fixtures.py on:
  * the reference's small real fixtures (refemu_fixtures.json), and
  * 720 seeded pairs of 20-200 bp (refemu_stage2.json); the 96 whose stage 2
    exits 0 with more than the end cell are kept, each labelled with how its list
    relates to the oracle's canonical traceback (tests/stage2_relations.py).

The CPU test re-derives every label with the oracle, so a label can never drift
from what the oracle says.  The GPU tests compare what swb_align_pair returns
with the reference's own lists, class by class:
  equal                the GPU list is the reference's list
  crosspoints_missed   same start and end; every reference crosspoint is one of
                       the GPU's (the reference's window search missed the rest)
  other_optimal_start  same end; the reference's start begins another alignment
                       of the same score, the GPU's is the canonical one
  start_not_found      same end; the reference printed no start; its crosspoints
                       lie on an optimal alignment to the GPU's end cell
  shipped_carry_end    the reference's stage 1 itself ended elsewhere (its
                       left-boundary carry); the GPU returns the textbook result
"""
import collections

import pytest

import oracle_ctypes as O
import swb200
from conftest import load_fixture_fasta, load_json
from stage2_relations import on_optimal_path, relation


def _cases():
    return load_json("refemu_stage2.json")


def test_stage2_labels_match_the_oracle():
    d = _cases()
    assert sum(d["outcomes"].values()) == d["pairs"]
    assert d["outcomes"]["listed"] == len(d["cases"])
    counts = collections.Counter()
    for c in d["cases"]:
        got = relation(c["a"].encode(), c["b"].encode(), c["scoring"], c["xpoints"])
        assert got == c["relation"], c
        counts[got] += 1
    assert dict(counts) == d["relations"]
    # the pinned classes are all present
    assert counts["equal"] >= 30 and counts["crosspoints_missed"] >= 30


def _check_against_reference(ctx, a: bytes, b: bytes, sc, ref, rel):
    ref = [tuple(x) for x in ref]
    r = ctx.align(a, b, swb200.scoring(*sc))
    got = [tuple(x) for x in r.xpoints]
    rows, cols, _ = O.orient(a, b)
    s = O.scoring(*sc)
    if rel == "shipped_carry_end":
        e = O.stage1(rows, cols, s, O.TEXTBOOK, O.TIE_REFERENCE)
        assert got[-1] == (e.row, e.col, e.score, 0)
        c = O.stage1(rows, cols, s, O.SHIPPED_CARRY, O.TIE_REFERENCE)
        assert ref[-1][:3] == (c.row, c.col, c.score)
        return
    assert got[-1] == ref[-1], (ref, got)
    if rel == "equal":
        assert got == ref
        return
    er, ec, best = got[-1][0], got[-1][1], got[-1][2]
    if rel == "crosspoints_missed":
        assert got[0] == ref[0]
        assert set(ref[1:-1]) <= set(got[1:-1]), (ref, got)
        return
    if rel == "other_optimal_start":
        assert ref[0][2] == 0 and got[0][2] == 0
        assert O.anchored_score(rows, cols, s, ref[0][0], ref[0][1], er, ec) == best
        assert O.anchored_score(rows, cols, s, got[0][0], got[0][1], er, ec) == best
        return
    assert rel == "start_not_found", rel
    assert got[0][2] == 0 and O.anchored_score(rows, cols, s, got[0][0], got[0][1], er, ec) == best
    for x in ref[:-1]:
        assert x in got or on_optimal_path(rows, cols, s, x, er, ec, best), (x, got)


@pytest.mark.gpu
def test_gpu_against_the_reference_stage2_sweep(gpu_ctx):
    seen = collections.Counter()
    for c in _cases()["cases"]:
        _check_against_reference(gpu_ctx, c["a"].encode(), c["b"].encode(), c["scoring"], c["xpoints"],
                                 c["relation"])
        seen[c["relation"]] += 1
    assert seen["equal"] >= 30


@pytest.mark.gpu
def test_gpu_against_the_reference_stage2_on_real_fixtures(gpu_ctx):
    """seq3/seq4: the reference's list equals the GPU's; seq0/seq1: same start and
    end, the reference's search missed the crosspoint between them; A00142/A00145:
    the reference printed the end cell only (its start search found nothing), with
    its stage-1 score, which its left-boundary carry inflates at the same cell."""
    checked = 0
    for f in load_json("refemu_fixtures.json"):
        s2 = f.get("stage2", {})
        if s2.get("exit_code") != 0 or not s2.get("xpoints"):
            continue
        a, b = load_fixture_fasta(f["a"]), load_fixture_fasta(f["b"])
        ref = [tuple(x) for x in s2["xpoints"]]
        if len(ref) == 1:
            # end cell only; the reference's own stage 1 scored it with its
            # left-boundary carry (520 where textbook Gotoh gives 480 at the same cell)
            rows, cols, _ = O.orient(a, b)
            s = O.scoring(*f["scoring"])
            c = O.stage1(rows, cols, s, O.SHIPPED_CARRY, O.TIE_REFERENCE)
            assert ref[0][:3] == (c.row, c.col, c.score)
            e = O.stage1(rows, cols, s, O.TEXTBOOK, O.TIE_REFERENCE)
            r = gpu_ctx.align(a, b, swb200.scoring(*f["scoring"]))
            assert tuple(r.xpoints[-1]) == (e.row, e.col, e.score, 0)
            assert (r.end_row, r.end_col) == ref[0][:2]
            checked += 1
            continue
        rel = relation(a, b, f["scoring"], ref)
        assert rel == {"0/seq0.fna.gz": "crosspoints_missed", "0/seq3.fna.gz": "equal"}[f["a"]], (f["a"], rel)
        _check_against_reference(gpu_ctx, a, b, f["scoring"], ref, rel)
        checked += 1
    assert checked == 3
