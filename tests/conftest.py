"""Shared test setup: paths, the `gpu` marker, fixture loaders."""
from __future__ import annotations

import gzip
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "projekt-2012_b200"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_fixture_fasta(rel: str) -> bytes:
    """Sequence bytes of a gzip'd reference FASTA fixture, read with the
    reference loader's rules (first line is the header; '\\n' and '\\r' dropped)."""
    data = gzip.open(os.path.join(GOLDEN, "seqs", rel), "rb").read()
    nl = data.find(b"\n")
    header_len = min(nl + 1 if nl >= 0 else len(data), 299)
    return data[header_len:].replace(b"\n", b"").replace(b"\r", b"")


def load_json(name: str):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def goldens():
    return load_json("goldens.json")


@pytest.fixture(scope="session")
def gpu_ctx():
    import swb200
    ctx = swb200.Context(device=0)
    yield ctx
    ctx.close()
