"""Serving loop (swb_server_*) on the GPU: requests of mixed length arrive while
others run, are admitted against the HBM budget and batched, and every result
is exactly the one the plain pair path gives the same pair alone."""
import random
import threading
import time

import pytest

import swb200

pytestmark = pytest.mark.gpu

SC = (1, -3, -5, -2)


def _pair(rng, n, sub=0.08):
    a = bytes(rng.choice(b"ACGT") for _ in range(n))
    lo = rng.randint(0, n // 4)
    core = bytearray(a[lo:lo + int(n * 0.7)])
    for i in range(len(core)):
        if rng.random() < sub:
            core[i] = rng.choice(b"ACGT")
    b = bytes(rng.choice(b"ACGT") for _ in range(rng.randint(0, n // 4))) + bytes(core)
    return (a, b) if rng.random() < 0.5 else (b, a)


def _same(x, y):
    return (x.score, x.end_row, x.end_col, x.start_row, x.start_col, x.swapped, x.ops, x.xpoints) == \
           (y.score, y.end_row, y.end_col, y.start_row, y.start_col, y.swapped, y.ops, y.xpoints)


def test_each_result_is_the_same_alone_and_in_the_mix(gpu_ctx):
    rng = random.Random(21)
    reqs = [_pair(rng, rng.randint(30, 2500)) for _ in range(160)]
    reqs += [_pair(rng, rng.randint(4000, 6000), sub=0.04) for _ in range(3)]   # long lane (long_cells below)
    reqs += [(b"", b"ACGT"), (b"ACGTACGT", b"TTTTGGGG")]
    rng.shuffle(reqs)
    ids, infos, results = [], {}, {}
    with swb200.Server(swb200.scoring(*SC), long_cells=10_000_000, hbm_budget_bytes=8 << 30) as srv:
        def submitter():
            for a, b in reqs:
                ids.append(srv.submit(a, b))
                time.sleep(rng.random() * 0.002)      # arrivals spread while earlier ones run
        th = threading.Thread(target=submitter)
        th.start()
        th.join()
        for k, rid in enumerate(ids):
            res, info = srv.wait(rid)
            results[k], infos[k] = res, info
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["long_completed"] == 3
    assert st["max_batch_seen"] > 1                       # short requests were batched
    assert any(i["lane"] == 1 for i in infos.values())
    for k, (a, b) in enumerate(reqs):
        alone = gpu_ctx.align(a, b, swb200.scoring(*SC))
        assert _same(results[k], alone), (k, len(a), len(b))


def test_burst_is_batched_and_budget_limits_admission(gpu_ctx):
    rng = random.Random(22)
    reqs = [_pair(rng, rng.randint(500, 1500)) for _ in range(120)]
    # a budget that holds only a few short requests at a time
    with swb200.Server(swb200.scoring(*SC), hbm_budget_bytes=4 << 20) as srv:
        ids = [srv.submit(a, b) for a, b in reqs]
        out = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert st["peak_reserved_bytes"] <= 4 << 20
    assert st["iterations"] >= 2
    for (a, b), (res, info) in zip(reqs, out):
        alone = gpu_ctx.align(a, b, swb200.scoring(*SC))
        assert _same(res, alone)
        assert info["total_ms"] >= info["run_ms"] >= 0


def test_request_larger_than_the_budget_is_refused():
    with swb200.Server(swb200.scoring(*SC), hbm_budget_bytes=1 << 20) as srv:
        with pytest.raises(swb200.SwbError) as ei:
            srv.submit(b"A" * 100_000, b"C" * 100_000)
        assert ei.value.code == swb200.SWB_ENOMEM_BUDGET
        with pytest.raises(swb200.SwbError) as ei:
            srv.wait(12345, 0)
        assert ei.value.code == swb200.SWB_ENOTFOUND


def test_wait_timeout_and_destroy_with_queued_requests():
    rng = random.Random(23)
    srv = swb200.Server(swb200.scoring(*SC))
    ids = [srv.submit(*_pair(rng, 3000)) for _ in range(50)]
    r = srv.wait(ids[0], 0)          # may or may not be done: either a result or None
    assert r is None or r[0].score >= 0
    srv.close()                      # queued requests are dropped, running ones finish


def test_serving_mix_stream_results_equal_the_plain_path(gpu_ctx):
    """A seeded stretch of the serving workload's own stream (synth.serving_stream:
    Poisson arrivals, 95% short pairs of 200-5,000 bp, 5% long pairs of 100 kbp -
    2 Mbp, scoring 1/-3/-5/-2, full traceback, 100 GB budget) submitted at its
    arrival times: every result, long or short, equals the plain path's on the
    same pair alone."""
    from swb200 import synth
    stream = synth.serving_stream(6.0, 12.0, seed_extra=7)
    assert any(lg for *_, lg in stream) and sum(1 for *_, lg in stream if not lg) > 40
    sc = swb200.scoring(*SC)
    ids = []
    with swb200.Server(sc, hbm_budget_bytes=100 << 30) as srv:
        start = time.perf_counter()
        for t_arr, q, tg, _ in stream:
            now = time.perf_counter() - start
            if t_arr > now:
                time.sleep(t_arr - now)
            ids.append(srv.submit(q, tg))
        got = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert st["completed"] == len(stream) and st["failed"] == 0
    with swb200.Context(device=0, hbm_budget_bytes=50 << 30) as ctx:
        for (t_arr, q, tg, lg), (res, info) in zip(stream, got):
            assert info["lane"] == (1 if lg else 0)
            alone = ctx.align(q, tg, sc)
            assert _same(res, alone), (len(q), len(tg), lg)
