"""The multi-process path on the CPU: two gloo ranks (subprocesses on
127.0.0.1) run the helpers bench.py and sharded batches use
(projekt-2012_b200/swb200/ranks.py): the slowest rank's time, the replicas'
whole-job rate, and a batch split by cell count whose per-rank oracle results,
gathered back in order, equal one process aligning the whole batch."""
import json
import os
import socket
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import ranks_worker as W  # noqa: E402
from swb200.ranks import gather_in_order, lpt_shards  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks(tmp_path):
    out = os.path.join(tmp_path, "rank0.json")
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, os.path.join(HERE, "ranks_worker.py"), out], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT))
    logs = []
    for p in procs:
        try:
            o, _ = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        logs.append(o.decode(errors="replace")[-2000:])
    assert all(p.returncode == 0 for p in procs), logs
    got = json.load(open(out))
    pairs = W.batch(5, 60)
    want = [list(W.align(p, (2, -3, -5, -2))) for p in pairs]
    assert got["results"] == want
    shards = got["shards"]
    assert sorted(i for s in shards for i in s) == list(range(len(pairs)))
    heaviest = max(len(a) * len(b) for a, b in pairs)
    assert abs(got["loads"][0] - got["loads"][1]) <= heaviest  # LPT balance bound


def test_lpt_shards_rules():
    w = [5, 9, 1, 9, 3, 7, 0]
    s = lpt_shards(w, 3)
    assert sorted(i for x in s for i in x) == list(range(len(w)))
    loads = [sum(w[i] for i in x) for x in s]
    assert max(loads) - min(loads) <= max(w)
    assert lpt_shards(w, 3) == s  # deterministic
    assert lpt_shards(w, 1) == [list(range(len(w)))]
    with pytest.raises(ValueError):
        lpt_shards(w, 0)


def test_gather_in_order_single_process():
    assert gather_in_order(["b", "a"], [1, 0], 2) == ["a", "b"]
    with pytest.raises(ValueError):
        gather_in_order(["a"], [0], 2)
