"""FASTA loading (swb_fasta_load, no GPU needed) and the CLI's error paths."""
import gzip
import os
import subprocess

import pytest

import swb200
from conftest import GOLDEN, load_fixture_fasta

CLI = os.path.join(os.path.dirname(swb200.LIB_PATH), "SWalign")
FIXTURES = sorted(os.path.join(d, f) for d in os.listdir(os.path.join(GOLDEN, "seqs"))
                  for f in os.listdir(os.path.join(GOLDEN, "seqs", d)))


@pytest.mark.parametrize("rel", FIXTURES)
def test_reference_rules_on_the_reference_inputs(rel, tmp_path):
    raw = gzip.open(os.path.join(GOLDEN, "seqs", rel), "rb").read()
    path = os.path.join(tmp_path, "in.fna")
    with open(path, "wb") as f:
        f.write(raw)
    [(name, seq)] = swb200.fasta_load(path)
    assert seq == load_fixture_fasta(rel)
    first = raw[:199].split(b"\n")[0] + b"\n"
    assert name.encode() == first[1:-1]


def test_multi_record_reader(tmp_path):
    long_header = "chr1 " + "x" * 400
    text = (f">{long_header}\r\nacgtNN\r\nAC GT\n;a comment\n\n>second record\nTTTT\n>empty\n").encode()
    path = os.path.join(tmp_path, "multi.fa")
    with open(path, "wb") as f:
        f.write(text)
    recs = swb200.fasta_load(path, swb200.FASTA_MULTI)
    assert recs == [(long_header, b"acgtNNACGT"), ("second record", b"TTTT"), ("empty", b"")]
    assert swb200.fasta_load(path, swb200.FASTA_MULTI | swb200.FASTA_UPPER)[0][1] == b"ACGTNNACGT"
    # the reference rules on the same file: one record, the long header spills into the sequence
    [(_, seq)] = swb200.fasta_load(path)
    assert seq == text[299:].replace(b"\n", b"").replace(b"\r", b"")


def test_load_errors(tmp_path):
    bad = os.path.join(tmp_path, "bad.fa")
    with open(bad, "wb") as f:
        f.write(b"ACGT\n")
    for p in (bad, os.path.join(tmp_path, "missing.fa")):
        for flags in (0, swb200.FASTA_MULTI):
            with pytest.raises(swb200.SwbError) as ei:
                swb200.fasta_load(p, flags)
            assert ei.value.code == swb200.SWB_EINVAL


def test_cli_argument_and_load_errors(tmp_path):
    r = subprocess.run([CLI, "a", "b"], capture_output=True, text=True)
    assert r.returncode == 255 and "Expected 6 input arguments, not 2!\n" in r.stdout
    r = subprocess.run([CLI, os.path.join(tmp_path, "none.fa"), "x", "1", "-3", "-5", "-2"], capture_output=True,
                       text=True)
    assert r.returncode == 255 and "ERROR\nAn error has occured while loading input sequences.\n" in r.stdout


@pytest.mark.gpu
def test_cli_result_line_matches_the_reference_golden(goldens, tmp_path):
    g = goldens[0]
    paths = []
    for rel in (g["a"], g["b"]):
        p = os.path.join(tmp_path, os.path.basename(rel)[:-3])
        with open(p, "wb") as f:
            f.write(gzip.open(os.path.join(GOLDEN, "seqs", rel), "rb").read())
        paths.append(p)
    sc = [str(v) for v in g["scoring"]]
    r = subprocess.run([CLI, *paths, *sc], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, SWB_GAP_LISTS=os.path.join(tmp_path, "gaps")))
    assert r.returncode == 0, r.stdout[-2000:]
    assert f"\t>Alignment score: {g['score']} at [{g['row1']}, {g['col1']}]\n\n" in r.stdout
    assert "Visual representation of the alignment" in r.stdout
    assert os.path.exists(os.path.join(tmp_path, "gaps.first.bin"))
