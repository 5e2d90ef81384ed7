"""The stage-1 autotuner (csrc/autotune.cpp): rows per lane chosen by timed
probes per shape bucket and kept in the file named by SWB_AUTOTUNE_CACHE.  The
reference hard-wires its launch shape (src/SWutils.cpp:233-253).  A first
process probes and appends the bucket's choice to the file; a second process
reads it back and appends nothing; every candidate gives the same result.
The packed batch pass is tuned the same way (448- or 256-row strips), its
probes timed on strided samples of the batch's own pairs."""
import json
import os
import random
import re
import subprocess
import sys

import pytest

import oracle_ctypes as O
import swb200

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _run(env):
    p = subprocess.run([sys.executable, os.path.join(HERE, "autotune_worker.py"), "1"], env=env,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_autotune_cache_file_round_trips(tmp_path):
    cache = str(tmp_path / "autotune.txt")
    env = {k: v for k, v in os.environ.items() if k != "SWB_STAGE1_R"}
    env["SWB_AUTOTUNE_CACHE"] = cache
    first = _run(env)
    lines = open(cache).read().splitlines()
    assert len(lines) == 1, lines
    key, R = lines[0].rsplit(" ", 1)
    assert key.startswith("sms") and " score " in key and int(R) in (8, 14, 16, 32)
    second = _run(env)          # reads the entry: no probe, nothing appended
    assert open(cache).read().splitlines() == lines
    assert second == first
    # a choice written by hand is used as it is
    other = 8 if int(R) != 8 else 16
    with open(cache, "w") as f:
        f.write(f"{key} {other}\n")
    assert _run(env) == first


def test_every_rows_per_lane_candidate_gives_the_same_result(gpu_ctx, monkeypatch):
    rng = random.Random(4)
    a = bytes(rng.choice(b"ACGT") for _ in range(40_000))
    b = bytes(c if rng.random() > 0.06 else rng.choice(b"ACGT") for c in a[5_000:25_000])
    rows, cols, _ = O.orient(a, b)
    e = O.stage1_fast(rows, cols, O.scoring(1, -3, -5, -2), O.TIE_REFERENCE)[0]
    for R in ("8", "14", "16", "32"):
        monkeypatch.setenv("SWB_STAGE1_R", R)
        for flags in (swb200.FLAG_SCORE_ONLY, 0):
            r = gpu_ctx.align(a, b, swb200.scoring(1, -3, -5, -2), flags)
            assert (r.score, r.end_row, r.end_col) == (e.score, e.row, e.col), (R, flags)


def _run_batch(env):
    p = subprocess.run([sys.executable, os.path.join(HERE, "autotune_worker.py"), "batch"], env=env,
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    m = re.search(r"packed rows per lane (\d+) \((\w+)\)", p.stderr)
    assert m, p.stderr
    return json.loads(p.stdout.strip().splitlines()[-1]), int(m.group(1)), m.group(2)


def test_batch_autotune_probes_once_and_the_cache_file_round_trips(tmp_path):
    """A first process probes both strip heights on samples of the 20,000-pair
    batch and records the bucket's choice; a second reads it and probes
    nothing; a choice written by hand is used; every run gives the same
    results, which equal the oracle's on a sample."""
    cache = str(tmp_path / "autotune.txt")
    env = {k: v for k, v in os.environ.items() if k not in ("SWB_BATCH16_R", "SWB_BATCH_PACK")}
    env["SWB_AUTOTUNE_CACHE"] = cache
    first, R1, how1 = _run_batch(env)
    assert how1 == "probed" and R1 in (8, 14)
    lines = open(cache).read().splitlines()
    assert len(lines) == 1 and " batch16 tab " in lines[0], lines
    key, R = lines[0].rsplit(" ", 1)
    assert int(R) == R1
    second, R2, how2 = _run_batch(env)
    assert (R2, how2) == (R1, "cached")
    assert open(cache).read().splitlines() == lines
    assert second == first
    other = 8 if R1 == 14 else 14
    with open(cache, "w") as f:
        f.write(f"{key} {other}\n")
    third, R3, how3 = _run_batch(env)
    assert (R3, how3) == (other, "cached")
    assert third == first
    # a sample against the oracle
    import autotune_worker as W
    from swb200 import synth
    buf, refs, sc = synth.batched(W.BATCH_PAIRS, seed_extra=5)
    buf = buf.tobytes()
    for i in random.Random(2).sample(range(W.BATCH_PAIRS), 30):
        qo, ql, to, tl = (int(x) for x in refs[i])
        rows, cols, _ = O.orient(buf[qo:qo + ql], buf[to:to + tl])
        e = O.stage1(rows, cols, O.scoring(*sc), O.TEXTBOOK, O.TIE_REFERENCE)
        assert (first["score"][i], first["end_row"][i], first["end_col"][i]) == (e.score, e.row, e.col), i
