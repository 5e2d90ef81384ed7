"""Generates tests/golden/chromosome_golden.json: the oracle's stage-1 result (score
and 0-based end cell under both tie rules) for the full chromosome-scale pair of
swb200.synth.chromosome_pair() (two ~10 Mbp sequences sharing an 8 Mbp ancestor,
about 10^14 cells, scoring 1/-3/-5/-2), with digests of the generated sequences so
that a change of the generator is caught.

Uses the oracle's AVX-512 wavefront (orc_stage1_simd, both tie rules in one pass):
about an hour on 8 host cores.  Run from the repository root after building the
oracle (make -C oracle):

    python tests/golden/make_chromosome_golden.py [threads]
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "projekt-2012_b200"))

import oracle_ctypes as O  # noqa: E402
from swb200 import synth  # noqa: E402


def main():
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    a, b, sc = synth.chromosome_pair()
    rows, cols, swapped = O.orient(a, b)
    out = {"generator": "swb200.synth.chromosome_pair()", "scoring": list(sc),
           "sha256_a": hashlib.sha256(a).hexdigest(), "sha256_b": hashlib.sha256(b).hexdigest(),
           "rows": len(rows), "cols": len(cols), "swapped": swapped}
    t0 = time.time()
    r = O.stage1_simd_both(rows, cols, O.scoring(*sc), threads=threads)
    if r is None:
        sys.exit("this CPU has no AVX-512; the scalar oracle would take about 13 hours")
    (ref, rowmajor), secs = r
    out["reference"] = {"score": ref.score, "end_row": ref.row, "end_col": ref.col}
    out["rowmajor"] = {"score": rowmajor.score, "end_row": rowmajor.row, "end_col": rowmajor.col}
    out["oracle"] = f"orc_stage1_simd, {threads} threads, {secs:.0f} s"
    print(out, f"{time.time() - t0:.0f} s", flush=True)
    with open(os.path.join(HERE, "chromosome_golden.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
