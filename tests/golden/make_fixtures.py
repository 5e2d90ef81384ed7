"""Generates the committed golden fixtures under tests/golden/.

Run from the repository root in a checkout that has the reference at
/root/reference and the reference's CPU build (make -C oracle ref):

    python tests/golden/make_fixtures.py

Outputs (all read by the tests; nothing reads /root/reference at test time):
  seqs/<set>/<file>.gz   the reference's FASTA inputs Sequences/0..5, gzip-compressed
  goldens.json           the expected score / 1-based end cell echoed by
                         Tests/test1.sh .. test5.sh (test6.sh names missing data
                         and repeats test4's line, so it is left out)
  refemu_cases.json      seeded random pairs with the reference build's score and
                         end cell (as-shipped stage 1, including its left-boundary
                         carry), used to pin the oracle's ORC_SHIPPED_CARRY mode
  refemu_fixtures.json   the reference build's stage-1 and stage-2 outcome on the
                         small real fixtures (score line, crosspoints, or the way
                         stage 2 failed: exit code / timeout)
  refemu_stage2.json     the reference build's stage 2 on seeded small pairs
                         (20-200 bp): every pair whose stage 2 exits 0 with a start
                         and an end cell, its crosspoint list, and how that list
                         relates to the oracle's canonical traceback; plus counts of
                         the ways the reference's stage 2 failed on the others

The reference checkout is read from $SWB_REFERENCE (default /root/reference).
`python tests/golden/make_fixtures.py stage2` regenerates refemu_stage2.json only.
"""
from __future__ import annotations

import gzip
import json
import multiprocessing
import os
import random
import re
import subprocess
import sys
import tempfile

REF = os.environ.get("SWB_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle_ctypes as O  # noqa: E402
from stage2_relations import relation  # noqa: E402


def copy_sequences():
    for d in sorted(os.listdir(os.path.join(REF, "Sequences"))):
        src_dir = os.path.join(REF, "Sequences", d)
        dst_dir = os.path.join(HERE, "seqs", d)
        os.makedirs(dst_dir, exist_ok=True)
        for f in sorted(os.listdir(src_dir)):
            data = open(os.path.join(src_dir, f), "rb").read()
            with gzip.GzipFile(os.path.join(dst_dir, f + ".gz"), "wb", compresslevel=9, mtime=0) as g:
                g.write(data)


def parse_goldens():
    out = []
    for i in range(1, 6):
        txt = open(os.path.join(REF, "Tests", f"test{i}.sh")).read()
        m = re.search(r"\./SWalign\s+(\S+)\s+(\S+)\s+(-?\d+)\s+(-?\d+)\s+(-?\d+)\s+(-?\d+)", txt)
        e = re.search(r"Alignment score should be: (\d+) at \[(\d+), (\d+)\]", txt)
        a, b = m.group(1), m.group(2)
        out.append({
            "test": f"Tests/test{i}.sh",
            "a": a.replace("Sequences/", "") + ".gz",
            "b": b.replace("Sequences/", "") + ".gz",
            "scoring": [int(m.group(k)) for k in range(3, 7)],
            "score": int(e.group(1)), "row1": int(e.group(2)), "col1": int(e.group(3)),
        })
    return out


def random_pair(rng):
    la = rng.choice([rng.randint(4, 30), rng.randint(20, 120), rng.randint(100, 300)])
    lb = rng.choice([rng.randint(4, 30), rng.randint(20, 120), rng.randint(100, 300)])
    alph = rng.choice(["ACGT", "AC", "A", "ACGTN"])
    a = "".join(rng.choice(alph) for _ in range(la))
    if rng.random() < 0.5:
        st = rng.randint(0, max(0, la - 1))
        b = list(a[st:st + lb]) or ["A"]
        for i in range(len(b)):
            if rng.random() < 0.1:
                b[i] = rng.choice(alph)
        b = "".join(b) + "".join(rng.choice(alph) for _ in range(max(0, lb - len(b))))
    else:
        b = "".join(rng.choice(alph) for _ in range(lb))
    sc = rng.choice([(1, -3, -5, -2), (5, -5, -5, -5), (2, -3, -5, -2), (1, -1, -1, -1), (3, -1, -2, -1)])
    return a, b, sc


def refemu_cases(n=240, seed=2012):
    rng = random.Random(seed)
    td = tempfile.mkdtemp()
    cases = []
    while len(cases) < n:
        a, b, sc = random_pair(rng)
        if min(len(a), len(b)) < 4:
            continue
        fa, fb = os.path.join(td, "a.fa"), os.path.join(td, "b.fa")
        open(fa, "w").write(">a\n" + a + "\n")
        open(fb, "w").write(">b\n" + b + "\n")
        r = O.run_reference(fa, fb, *sc, stage1_only=True, timeout=60)
        cases.append({"a": a, "b": b, "scoring": list(sc),
                      "score": r["score"], "row1": r["row1"], "col1": r["col1"],
                      "G": r["G"], "T": r["T"], "P1": r["P1"], "P2": r["P2"]})
    return cases


def refemu_fixture_runs():
    runs = []
    pairs = [("1/A00142.fna", "1/A00145.fna", (5, -5, -5, -5)),
             ("2/NC_005046.fna", "2/NC_012557.fna", (5, -5, -5, -5)),
             ("0/seq0.fna", "0/seq1.fna", (5, -5, -5, -5)),
             ("0/seq5.fna", "0/seq6.fna", (1, -3, -5, -2)),
             ("0/seq3.fna", "0/seq4.fna", (1, -3, -5, -2))]
    for fa, fb, sc in pairs:
        pa, pb = os.path.join(REF, "Sequences", fa), os.path.join(REF, "Sequences", fb)
        s1 = O.run_reference(pa, pb, *sc, stage1_only=True, timeout=120)
        entry = {"a": fa + ".gz", "b": fb + ".gz", "scoring": list(sc),
                 "score": s1["score"], "row1": s1["row1"], "col1": s1["col1"]}
        try:
            s2 = O.run_reference(pa, pb, *sc, stage1_only=False, timeout=30)
            entry["stage2"] = {"exit_code": s2["rc"], "xpoints": s2["xpoints"]}
        except subprocess.TimeoutExpired:
            entry["stage2"] = {"timeout_s": 30}
        runs.append(entry)
    return runs


def _mutate(rng, s, alph, sub, indel):
    out, i = [], 0
    while i < len(s):
        r = rng.random()
        if r < indel / 2:
            out.append(rng.choice(alph))
            continue
        if r < indel:
            i += 1
            continue
        out.append(rng.choice(alph) if rng.random() < sub else s[i])
        i += 1
    return "".join(out)


def stage2_pair(rng):
    """A small pair for the stage-2 sweep: 70% a mutated window of A inside random
    padding (so that there is an alignment crossing several special rows), 30%
    unrelated sequences; both at least 20 bp (the reference's full launch shape)."""
    alph = rng.choice(["ACGT", "ACGT", "ACGT", "AC"])
    la = rng.randint(20, 200)
    a = "".join(rng.choice(alph) for _ in range(la))
    if rng.random() < 0.7:
        st = rng.randint(0, la // 3)
        ln = rng.randint(la // 3, la - st)
        core = _mutate(rng, a[st:st + ln], alph, rng.choice([0.0, 0.03, 0.08]), rng.choice([0.0, 0.01, 0.03]))
        b = "".join(rng.choice(alph) for _ in range(rng.randint(0, 30))) + core + \
            "".join(rng.choice(alph) for _ in range(rng.randint(0, 30)))
    else:
        b = "".join(rng.choice(alph) for _ in range(rng.randint(20, 200)))
    if len(b) < 20:
        b += "".join(rng.choice(alph) for _ in range(20 - len(b)))
    sc = rng.choice([(1, -3, -5, -2), (5, -5, -5, -5), (2, -3, -5, -2), (1, -1, -1, -1), (3, -1, -2, -1)])
    return a, b, sc


def _stage2_run(job):
    i, a, b, sc = job
    td = tempfile.mkdtemp()
    fa, fb = os.path.join(td, "a.fa"), os.path.join(td, "b.fa")
    with open(fa, "w") as f:
        f.write(">a\n" + a + "\n")
    with open(fb, "w") as f:
        f.write(">b\n" + b + "\n")
    try:
        r = O.run_reference(fa, fb, *sc, stage1_only=False, timeout=10)
    except subprocess.TimeoutExpired:
        return i, "timeout", None
    if r["rc"] != 0:
        return i, f"exit_{r['rc'] & 0xff}", None
    if len(r["xpoints"]) < 2:
        return i, "end_only", None
    return i, "listed", [list(x) for x in r["xpoints"]]


def refemu_stage2_sweep(n=720, seed=2012):
    rng = random.Random(seed)
    jobs = [(i,) + stage2_pair(rng) for i in range(n)]
    with multiprocessing.Pool(os.cpu_count()) as pool:
        results = pool.map(_stage2_run, jobs)
    counts, cases = {}, []
    for (i, kind, xps), (_, a, b, sc) in zip(results, jobs):
        counts[kind] = counts.get(kind, 0) + 1
        if kind == "listed":
            cases.append({"a": a, "b": b, "scoring": list(sc), "xpoints": xps,
                          "relation": relation(a.encode(), b.encode(), sc, xps)})
    rel = {}
    for c in cases:
        rel[c["relation"]] = rel.get(c["relation"], 0) + 1
    return {"pairs": n, "seed": seed, "outcomes": counts, "relations": rel, "cases": cases}


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "stage2":
        with open(os.path.join(HERE, "refemu_stage2.json"), "w") as f:
            json.dump(refemu_stage2_sweep(), f)
        print("refemu_stage2.json written to", HERE)
        return
    copy_sequences()
    with open(os.path.join(HERE, "goldens.json"), "w") as f:
        json.dump(parse_goldens(), f, indent=1)
    with open(os.path.join(HERE, "refemu_cases.json"), "w") as f:
        json.dump(refemu_cases(), f)
    with open(os.path.join(HERE, "refemu_fixtures.json"), "w") as f:
        json.dump(refemu_fixture_runs(), f, indent=1)
    with open(os.path.join(HERE, "refemu_stage2.json"), "w") as f:
        json.dump(refemu_stage2_sweep(), f)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
