"""Generates tests/golden/long_pair_golden.json: the oracle's stage-1 result (score
and 0-based end cell, both tie rules) for the full 1 Mbp long pair of
swb200.synth.long_pair() (1,000,000 x 999,837 cells, scoring 1/-3/-5/-2), with a
digest of the generated sequences so that a change of the generator is caught.

The oracle's multithreaded wavefront takes about 7 minutes per tie rule on 8 host
cores.  Run from the repository root after building the oracle (make -C oracle):

    python tests/golden/make_long_pair_golden.py
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
    a, b, sc = synth.long_pair()
    rows, cols, swapped = O.orient(a, b)
    out = {"generator": "swb200.synth.long_pair()", "scoring": list(sc),
           "sha256_a": hashlib.sha256(a).hexdigest(), "sha256_b": hashlib.sha256(b).hexdigest(),
           "rows": len(rows), "cols": len(cols), "swapped": swapped}
    for name, tie in (("reference", O.TIE_REFERENCE), ("rowmajor", O.TIE_ROWMAJOR)):
        t0 = time.time()
        r, _ = O.stage1_mt(rows, cols, O.scoring(*sc), tie, threads=os.cpu_count())
        out[name] = {"score": r.score, "end_row": r.row, "end_col": r.col}
        print(name, out[name], f"{time.time() - t0:.0f} s", flush=True)
    with open(os.path.join(HERE, "long_pair_golden.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
