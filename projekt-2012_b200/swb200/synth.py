"""Seeded synthetic DNA for the five workloads (no public dataset is named for
this path; these generators stand in with the stated shapes, sizes and rates).

RNG: numpy PCG64 seeded with 2012 + workload index.  Bases iid uniform over
{A,C,G,T}; a substitution replaces a base with one of the other three; an indel
event happens per source position with the given rate, half insertions of
random bases and half deletions, lengths geometric with the given mean.
"""
from __future__ import annotations

import numpy as np

BASES = np.frombuffer(b"ACGT", dtype=np.uint8)


def rng_for(workload: int, extra: int = 0) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64([2012 + workload, extra]))


def random_dna(rng: np.random.Generator, n: int) -> np.ndarray:
    return BASES[rng.integers(0, 4, size=n)]


def mutate(rng: np.random.Generator, src: np.ndarray, sub_rate: float, indel_rate: float,
           indel_mean: float) -> np.ndarray:
    s = src.copy()
    n = len(s)
    subs = np.nonzero(rng.random(n) < sub_rate)[0]
    if len(subs):
        codes = np.searchsorted(BASES, s[subs])
        s[subs] = BASES[(codes + rng.integers(1, 4, size=len(subs))) % 4]
    events = np.nonzero(rng.random(n) < indel_rate)[0]
    if len(events) == 0:
        return s
    kinds = rng.random(len(events)) < 0.5          # True: insertion
    lens = rng.geometric(1.0 / indel_mean, size=len(events))
    parts = []
    pos = 0
    for e, ins, L in zip(events.tolist(), kinds.tolist(), lens.tolist()):
        if e < pos:
            continue                                    # inside a previous deletion
        parts.append(s[pos:e])
        if ins:
            parts.append(random_dna(rng, L))
            pos = e
        else:
            pos = e + L
    parts.append(s[pos:])
    return np.concatenate(parts)


def plain_small(seed_extra: int = 0):
    """2,000 bp vs 400 + mutate(1,200-bp window, 10% sub, 2% indel, mean 3) + 400."""
    rng = rng_for(0, seed_extra)
    a = random_dna(rng, 2000)
    w = int(rng.integers(0, 2000 - 1200 + 1))
    core = mutate(rng, a[w:w + 1200], 0.10, 0.02, 3.0)
    b = np.concatenate([random_dna(rng, 400), core, random_dna(rng, 400)])
    return a.tobytes(), b.tobytes(), (1, -3, -5, -2)


def long_pair(length: int = 1_000_000, seed_extra: int = 0):
    """1 Mbp iid; B = mutate(central 80%, 5% sub, 1% indel, mean 4) with 10% random
    flanks on each side (100 kbp at the default length)."""
    rng = rng_for(1, seed_extra)
    a = random_dna(rng, length)
    lo, hi = length // 10, length - length // 10
    core = mutate(rng, a[lo:hi], 0.05, 0.01, 4.0)
    b = np.concatenate([random_dna(rng, lo), core, random_dna(rng, length - hi)])
    return a.tobytes(), b.tobytes(), (1, -3, -5, -2)


def chromosome_pair(ancestor: int = 8_000_000, flank: int = 1_000_000, seed_extra: int = 0):
    """Two ~10 Mbp sequences: independent mutate(ancestor, 3% sub, 0.5% indel, mean 4)
    with random flanks on both ends."""
    rng = rng_for(2, seed_extra)
    anc = random_dna(rng, ancestor)
    a = np.concatenate([random_dna(rng, flank), mutate(rng, anc, 0.03, 0.005, 4.0), random_dna(rng, flank)])
    b = np.concatenate([random_dna(rng, flank), mutate(rng, anc, 0.03, 0.005, 4.0), random_dna(rng, flank)])
    return a.tobytes(), b.tobytes(), (1, -3, -5, -2)


def batched(npairs: int = 100_000, seed_extra: int = 0, sigma: float = 0.75):
    """Batched workload: query lengths clip(round(lognormal(ln 1000, sigma)), 100,
    10,000); each target is 1.5x its query long, built from mutate(query, 8% sub,
    1% indel, mean 3) placed at a uniform random offset inside random padding.
    Returns (buffer, refs, scoring): one uint8 buffer holding every query and
    target, refs[i] = (query_off, query_len, target_off, target_len)."""
    rng = rng_for(3, seed_extra)
    q = np.clip(np.round(rng.lognormal(np.log(1000.0), sigma, size=npairs)), 100, 10_000).astype(np.int64)
    parts, refs, off = [], np.zeros((npairs, 4), dtype=np.int64), 0
    for i, L in enumerate(q.tolist()):
        query = random_dna(rng, L)
        core = mutate(rng, query, 0.08, 0.01, 3.0)
        tlen = int(round(1.5 * L))
        if len(core) > tlen:
            core = core[:tlen]
        pad = tlen - len(core)
        left = int(rng.integers(0, pad + 1))
        target = np.concatenate([random_dna(rng, left), core, random_dna(rng, pad - left)])
        refs[i] = (off, L, off + L, tlen)
        parts.append(query)
        parts.append(target)
        off += L + tlen
    return np.concatenate(parts), refs, (2, -3, -5, -2)


def serving_request(rng: np.random.Generator):
    """One request of the serving mix: 95% short pairs (query uniform 200-5,000 bp,
    target 1.5x built from the query with 7% substitutions and 1% indels, mean 3,
    inside random padding) and 5% long pairs (query uniform 100 kbp-2 Mbp, target
    1.5x with 2.5% substitutions and 0.5% indels, mean 4).  Returns (query, target,
    is_long)."""
    long = rng.random() < 0.05
    if long:
        L = int(rng.integers(100_000, 2_000_001))
        sub, indel, mean = 0.025, 0.005, 4.0
    else:
        L = int(rng.integers(200, 5_001))
        sub, indel, mean = 0.07, 0.01, 3.0
    query = random_dna(rng, L)
    core = mutate(rng, query, sub, indel, mean)
    tlen = int(round(1.5 * L))
    core = core[:tlen]
    pad = tlen - len(core)
    left = int(rng.integers(0, pad + 1))
    target = np.concatenate([random_dna(rng, left), core, random_dna(rng, pad - left)])
    return query.tobytes(), target.tobytes(), long


def serving_stream(duration_s: float, rate: float, seed_extra: int = 0):
    """Poisson arrivals at `rate` per second for duration_s seconds: list of
    (arrival time s, query, target, is_long)."""
    rng = rng_for(4, seed_extra)
    t, out = 0.0, []
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration_s:
            return out
        q, tg, lg = serving_request(rng)
        out.append((t, q, tg, lg))


def tall_pair(rows: int = 10_000_000, cols: int = 100_000, seed_extra: int = 0):
    """Profiling shape: `rows` iid bases against a mutated `cols`-long window of
    them (5% sub, 1% indel, mean 4); scoring 1/-3/-5/-2."""
    rng = rng_for(2, 1000 + seed_extra)
    a = random_dna(rng, rows)
    lo = rows // 2
    b = mutate(rng, a[lo:lo + cols], 0.05, 0.01, 4.0)
    return a.tobytes(), b.tobytes(), (1, -3, -5, -2)
