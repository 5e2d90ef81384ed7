"""The C ABI boundary without a GPU: the library loads, exports every function
include/swb200.h declares, and its host-only calls behave like the reference
(initScoringValues, getLaunchConfig + padding).  No compute call is made here."""
import os
import re
import subprocess

import pytest

import oracle_ctypes as O
import swb200
from conftest import ROOT


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "swb200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(swb_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_function():
    names = declared_functions()
    assert len(names) >= 10
    lib = swb200.lib()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_product_library_does_not_link_the_oracle():
    out = subprocess.run(["ldd", swb200.LIB_PATH], capture_output=True, text=True).stdout
    assert "oracle" not in out
    nm = subprocess.run(["nm", "-D", swb200.LIB_PATH], capture_output=True, text=True).stdout
    assert "orc_" not in nm


@pytest.mark.parametrize("args,ok", [
    (("1", "-3", "-5", "-2"), True), (("5", "-5", "-5", "-5"), True),
    (("0", "-3", "-5", "-2"), False), (("1", "0", "-5", "-2"), False),
    (("1", "-3", "0", "-2"), False), (("1", "-3", "-5", "1"), False),
    (("abc", "-3", "-5", "-2"), False), (("2x", "-3y", "-5", "-2"), True),
])
def test_scoring_parse_like_initScoringValues(args, ok):
    sc = swb200.Scoring()
    rc = swb200.lib().swb_scoring_parse(*[a.encode() for a in args], sc)
    assert (rc == swb200.SWB_OK) == ok
    if ok:
        assert (sc.match, sc.mismatch) == (int(re.match(r"-?\d+", args[0]).group()),
                                           int(re.match(r"-?\d+", args[1]).group()))


def test_reference_geometry_matches_oracle():
    for rows in (4, 9, 12, 19, 20, 21, 100, 1351, 1389, 2001, 10 ** 6 + 3):
        for cols in (3, 4, 5, 8, 9, 10, 11, 19, 20, 21, 99, 1000, 1351):
            if cols > rows:
                continue
            rc, G, T, P1, P2 = swb200.reference_geometry(rows, cols)
            g = O.geometry(rows, cols)
            assert (G, T, P1, P2) == (g.G, g.T, g.P1, g.P2)
            assert (rc == swb200.SWB_OK) == (g.T > 0)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_context_without_device_reports_cuda_error():
    with pytest.raises(swb200.SwbError) as e:
        swb200.Context(device=0)
    assert e.value.code == swb200.SWB_ECUDA


def test_cli_argument_count_and_load_errors(tmp_path):
    r = subprocess.run([swb200.CLI_PATH, "a"], capture_output=True, text=True)
    assert r.returncode == 255
    assert "Expected 6 input arguments, not 1!\n\n" in r.stdout
    bad = tmp_path / "bad.fa"
    bad.write_text("no header\nACGT\n")
    r = subprocess.run([swb200.CLI_PATH, str(bad), str(bad), "1", "-3", "-5", "-2"],
                       capture_output=True, text=True)
    assert r.returncode == 255
    assert "ERROR\nAn error has occured while loading input sequences.\n\n" in r.stdout
