"""One process of tests/test_autotune_gpu.py: aligns a seeded pair large enough
for the autotuner (score only), or with "batch" the seeded 20,000-pair batch
(packed pass, log on stderr), and prints the result as JSON."""
import json
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "projekt-2012_b200"))

import swb200  # noqa: E402


def pair():
    rng = random.Random(int(sys.argv[1]) if len(sys.argv) > 1 else 1)
    a = bytes(rng.choice(b"ACGT") for _ in range(210_000))
    core = bytearray(a[50_000:150_000])
    for i in range(0, len(core), 17):
        core[i] = rng.choice(b"ACGT")
    return a, bytes(core)


def batch():
    import numpy as np
    from swb200 import synth
    buf, refs, sc = synth.batched(BATCH_PAIRS, seed_extra=5)
    with swb200.Context(device=0, verbose=1) as ctx:
        r = ctx.batch_align(buf.tobytes(), refs, swb200.scoring(*sc), 0, trace_frac=0.0)
    print(json.dumps({"score": np.asarray(r.score).tolist(), "end_row": np.asarray(r.end_row).tolist(),
                      "end_col": np.asarray(r.end_col).tolist()}))


BATCH_PAIRS = 20_000

if __name__ == "__main__" and len(sys.argv) > 1 and sys.argv[1] == "batch":
    batch()
elif __name__ == "__main__":
    a, b = pair()
    with swb200.Context(device=0) as ctx:
        r = ctx.align(a, b, swb200.scoring(1, -3, -5, -2), swb200.FLAG_SCORE_ONLY)
    print(json.dumps({"score": r.score, "end": [r.end_row, r.end_col]}))
