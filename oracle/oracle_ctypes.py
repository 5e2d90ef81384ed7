"""ctypes access to the CPU oracle (oracle/build/liboracle.so) and to the CPU
build of the reference (oracle/_ref/swalign_emu).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs, never by the product.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess
from dataclasses import dataclass

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboracle.so")
REFEMU_PATH = os.path.join(HERE, "_ref", "swalign_emu")
VISUAL_PATH = os.path.join(HERE, "_ref", "visual_emu")

TEXTBOOK, SHIPPED_CARRY = 0, 1
TIE_REFERENCE, TIE_ROWMAJOR, TIE_BOTH = 0, 1, 2


class Scoring(C.Structure):
    _fields_ = [("match", C.c_int32), ("mismatch", C.c_int32),
                ("gap_open", C.c_int32), ("gap_extend", C.c_int32)]


class Geom(C.Structure):
    _fields_ = [("G", C.c_int32), ("T", C.c_int32), ("P1", C.c_int64),
                ("P2", C.c_int64), ("C", C.c_int64)]


class End(C.Structure):
    _fields_ = [("score", C.c_int32), ("row", C.c_int64), ("col", C.c_int64)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "build/liboracle.so"], check=True,
                           stdout=subprocess.DEVNULL)
        L = C.CDLL(LIB_PATH)
        u8p = C.c_char_p
        L.orc_geometry.argtypes = [C.c_int64, C.c_int64, C.POINTER(Geom)]
        L.orc_geometry.restype = C.c_int
        L.orc_tie_key.argtypes = [C.POINTER(Geom), C.c_int, C.c_int64, C.c_int64]
        L.orc_tie_key.restype = C.c_uint64
        L.orc_stage1.argtypes = [u8p, C.c_int64, u8p, C.c_int64, C.POINTER(Scoring),
                                 C.c_int, C.c_int, C.POINTER(End)]
        L.orc_stage1.restype = C.c_int
        L.orc_stage1_mt.argtypes = [u8p, C.c_int64, u8p, C.c_int64, C.POINTER(Scoring),
                                    C.c_int, C.c_int, C.POINTER(End), C.POINTER(C.c_int64)]
        L.orc_stage1_mt.restype = C.c_int
        L.orc_stage1_simd.argtypes = L.orc_stage1_mt.argtypes
        L.orc_stage1_simd.restype = C.c_int
        L.orc_special_rows.argtypes = [u8p, C.c_int64, u8p, C.c_int64, C.POINTER(Scoring),
                                       C.c_int64, C.c_void_p, C.c_int64]
        L.orc_special_rows.restype = C.c_int64
        L.orc_traceback.argtypes = [u8p, C.c_int64, u8p, C.c_int64, C.POINTER(Scoring),
                                    C.c_int64, C.c_int64, C.c_char_p, C.c_int64,
                                    C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.orc_traceback.restype = C.c_int64
        L.orc_traceback_xp.argtypes = [u8p, C.c_int64, u8p, C.c_int64, C.POINTER(Scoring),
                                       C.c_int64, C.c_int64, C.c_char_p, C.c_int64,
                                       C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                       C.c_int64, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]
        L.orc_traceback_xp.restype = C.c_int64
        L.orc_score_ops.argtypes = [u8p, u8p, C.POINTER(Scoring), C.c_int64, C.c_int64,
                                    C.c_char_p, C.c_int64]
        L.orc_score_ops.restype = C.c_int64
        L.orc_anchored_score.argtypes = [u8p, C.c_int64, u8p, C.c_int64, C.POINTER(Scoring),
                                         C.c_int64, C.c_int64, C.c_int64, C.c_int64]
        L.orc_anchored_score.restype = C.c_int64
        L.orc_block.argtypes = [u8p, C.c_int64, u8p, C.c_int64, C.POINTER(Scoring), C.c_void_p, C.c_void_p,
                                C.c_int32, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_void_p,
                                C.c_void_p, C.POINTER(End), C.POINTER(C.c_uint64)]
        L.orc_block.restype = C.c_int
        _lib = L
    return _lib


def scoring(match, mismatch, gap_open, gap_extend) -> Scoring:
    return Scoring(match, mismatch, gap_open, gap_extend)


def orient(a: bytes, b: bytes):
    """Longer sequence on rows; equal lengths keep argument order (SWutils.cpp:84-88)."""
    if len(a) < len(b):
        return b, a, True
    return a, b, False


def geometry(rows: int, cols: int) -> Geom:
    g = Geom()
    lib().orc_geometry(rows, cols, C.byref(g))
    return g


@dataclass
class Stage1:
    score: int
    row: int
    col: int


def stage1(rows: bytes, cols: bytes, sc: Scoring, semantics=TEXTBOOK, tie=TIE_REFERENCE) -> Stage1:
    e = End()
    rc = lib().orc_stage1(rows, len(rows), cols, len(cols), C.byref(sc), semantics, tie, C.byref(e))
    if rc != 0:
        raise RuntimeError(f"orc_stage1 failed: {rc}")
    return Stage1(e.score, e.row, e.col)


def stage1_mt(rows: bytes, cols: bytes, sc: Scoring, tie=TIE_REFERENCE, threads=None):
    """Returns (Stage1, seconds)."""
    threads = threads or os.cpu_count() or 1
    e = End()
    ns = C.c_int64(0)
    rc = lib().orc_stage1_mt(rows, len(rows), cols, len(cols), C.byref(sc), tie, threads,
                             C.byref(e), C.byref(ns))
    if rc != 0:
        raise RuntimeError(f"orc_stage1_mt failed: {rc}")
    return Stage1(e.score, e.row, e.col), ns.value * 1e-9


def stage1_simd(rows: bytes, cols: bytes, sc: Scoring, tie=TIE_REFERENCE, threads=None):
    """Returns (Stage1, seconds) from the AVX-512 wavefront, or None when the CPU
    has no AVX-512."""
    threads = threads or os.cpu_count() or 1
    e = End()
    ns = C.c_int64(0)
    rc = lib().orc_stage1_simd(rows, len(rows), cols, len(cols), C.byref(sc), tie, threads,
                               C.byref(e), C.byref(ns))
    if rc == -4:
        return None
    if rc != 0:
        raise RuntimeError(f"orc_stage1_simd failed: {rc}")
    return Stage1(e.score, e.row, e.col), ns.value * 1e-9


def stage1_simd_both(rows: bytes, cols: bytes, sc: Scoring, threads=None):
    """Both tie rules in one AVX-512 pass: ((reference, rowmajor), seconds) or None."""
    threads = threads or os.cpu_count() or 1
    e = (End * 2)()
    ns = C.c_int64(0)
    rc = lib().orc_stage1_simd(rows, len(rows), cols, len(cols), C.byref(sc), TIE_BOTH, threads,
                               e, C.byref(ns))
    if rc == -4:
        return None
    if rc != 0:
        raise RuntimeError(f"orc_stage1_simd failed: {rc}")
    return (Stage1(e[0].score, e[0].row, e[0].col), Stage1(e[1].score, e[1].row, e[1].col)), ns.value * 1e-9


def stage1_fast(rows: bytes, cols: bytes, sc: Scoring, tie=TIE_REFERENCE, threads=None):
    """The fastest multithreaded stage 1 this CPU runs: (Stage1, seconds, kind)."""
    r = stage1_simd(rows, cols, sc, tie, threads)
    if r is not None:
        return r[0], r[1], "avx512"
    s, t = stage1_mt(rows, cols, sc, tie, threads)
    return s, t, "scalar"


def special_rows(rows: bytes, cols: bytes, sc: Scoring, k: int):
    import numpy as np
    nrows = len(rows) // k
    out = np.zeros((max(nrows, 1), len(cols), 2), dtype=np.int32)
    got = lib().orc_special_rows(rows, len(rows), cols, len(cols), C.byref(sc), k,
                                 out.ctypes.data, nrows)
    return out[:got]


def traceback(rows: bytes, cols: bytes, sc: Scoring, er: int, ec: int):
    """Returns (ops:str, start_row, start_col)."""
    cap = len(rows) + len(cols) + 8
    buf = C.create_string_buffer(cap)
    sr, scol = C.c_int64(0), C.c_int64(0)
    k = lib().orc_traceback(rows, len(rows), cols, len(cols), C.byref(sc), er, ec, buf, cap,
                            C.byref(sr), C.byref(scol))
    if k < 0:
        raise RuntimeError(f"orc_traceback failed: {k}")
    return buf.raw[:k].decode(), sr.value, scol.value


def traceback_xp(rows: bytes, cols: bytes, sc: Scoring, er: int, ec: int, interval: int):
    """Returns (ops, start_row, start_col, [(row, col, score, gap), ...] top to bottom)."""
    import numpy as np
    cap = len(rows) + len(cols) + 8
    buf = C.create_string_buffer(cap)
    sr, scol, nx = C.c_int64(0), C.c_int64(0), C.c_int64(0)
    xcap = len(rows) // max(1, interval) + 8
    xs = np.zeros(4 * xcap, dtype=np.int64)
    k = lib().orc_traceback_xp(rows, len(rows), cols, len(cols), C.byref(sc), er, ec, buf, cap,
                               C.byref(sr), C.byref(scol), interval, xs.ctypes.data, xcap, C.byref(nx))
    if k < 0:
        raise RuntimeError(f"orc_traceback_xp failed: {k}")
    xps = [tuple(int(v) for v in xs[4 * i:4 * i + 4]) for i in range(nx.value)]
    return buf.raw[:k].decode(), sr.value, scol.value, xps


def score_ops(rows: bytes, cols: bytes, sc: Scoring, sr: int, scol: int, ops: str) -> int:
    o = ops.encode()
    return lib().orc_score_ops(rows, cols, C.byref(sc), sr, scol, o, len(o))


def anchored_score(rows: bytes, cols: bytes, sc: Scoring, sr: int, scol: int, er: int, ec: int) -> int:
    """Best score of an alignment from the diagonal cell (sr, scol) to (er, ec)."""
    return lib().orc_anchored_score(rows, len(rows), cols, len(cols), C.byref(sc), sr, scol, er, ec)


def block(rows: bytes, cols: bytes, sc: Scoring, top, left, corner: int, r0: int, c0: int,
          full_m: int, full_n: int, tie=TIE_REFERENCE):
    """One block of a chain (orc_block): returns (bottom, right, Stage1 best, key);
    top / left / bottom / right are int32 numpy arrays of shape (len, 2) or None."""
    import numpy as np
    m, n = len(rows), len(cols)
    bottom = np.zeros((n, 2), dtype=np.int32)
    right = np.zeros((m, 2), dtype=np.int32)
    t = None if top is None else np.ascontiguousarray(top, dtype=np.int32)
    lf = None if left is None else np.ascontiguousarray(left, dtype=np.int32)
    e, key = End(), C.c_uint64(0)
    rc = lib().orc_block(rows, m, cols, n, C.byref(sc), None if t is None else t.ctypes.data,
                         None if lf is None else lf.ctypes.data, corner, r0, c0, full_m, full_n, tie,
                         bottom.ctypes.data, right.ctypes.data, C.byref(e), C.byref(key))
    if rc != 0:
        raise RuntimeError(f"orc_block failed: {rc}")
    return bottom, right, Stage1(e.score, e.row, e.col), key.value


def crosspoints(ops: str, sr: int, scol: int, interval: int):
    """Rows where the path leaves a special row (0-based R = interval*k - 1) going
    down: returns [(row, col)] for each special row the path crosses, top to bottom."""
    out = []
    r, c = sr, scol
    path = [(r, c)]
    for o in ops[1:]:
        if o == "M":
            r += 1; c += 1
        elif o == "I":
            c += 1
        else:
            r += 1
        path.append((r, c))
    last_in_row = {}
    for (pr, pc) in path:
        last_in_row[pr] = pc
    er = path[-1][0]
    R = interval - 1
    while R < er:
        if R in last_in_row and R >= sr:
            out.append((R, last_in_row[R]))
        R += interval
    return out


def run_reference(fa: str, fb: str, match: int, mismatch: int, gap_open: int, gap_extend: int,
                  stage1_only=True, timeout=600):
    """Runs the CPU build of the reference; returns dict with score/row1/col1/geom/xpoints
    or raises subprocess.TimeoutExpired / RuntimeError."""
    if not os.path.exists(REFEMU_PATH):
        raise FileNotFoundError(REFEMU_PATH)
    args = [REFEMU_PATH, fa, fb, str(match), str(mismatch), str(gap_open), str(gap_extend)]
    if stage1_only:
        args.append("--stage1-only")
    p = subprocess.run(args, stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, timeout=timeout)
    res = {"rc": p.returncode, "xpoints": []}
    for line in p.stderr.decode(errors="replace").splitlines():
        f = line.split()
        if len(f) >= 2 and f[0] == "REFEMU":
            if f[1] == "score":
                res["score"], res["row1"], res["col1"] = int(f[2]), int(f[3]), int(f[4])
            elif f[1] == "geom":
                res["G"], res["T"], res["P1"], res["P2"] = map(int, f[2:6])
            elif f[1] == "xpoint":
                res["xpoints"].append(tuple(int(x) for x in f[3:7]))
    return res


def run_reference_visual(first: bytes, second: bytes, first_gaps: str, second_gaps: str, start, end,
                         timeout=60) -> str:
    """The reference's own renderer (src/Visualisation.cpp:11-129, built by
    `make ref` as _ref/visual_emu) on gap-list files: returns its stdout.  Each
    gap file gets one terminating record {-1, 0} appended first: the renderer
    reads its gap lists without an end check (Visualisation.cpp:68,88)."""
    import tempfile
    if not os.path.exists(VISUAL_PATH):
        raise FileNotFoundError(VISUAL_PATH)
    td = tempfile.mkdtemp()
    paths = []
    for k, (seq, gp) in enumerate(((first, first_gaps), (second, second_gaps))):
        sp = os.path.join(td, f"seq{k}.bin")
        with open(sp, "wb") as f:
            f.write(seq)
        g = os.path.join(td, f"gaps{k}.bin")
        with open(gp, "rb") as src, open(g, "wb") as dst:
            dst.write(src.read())
            dst.write(struct.pack("<ii", -1, 0))
        paths += [sp, g]
    p = subprocess.run([VISUAL_PATH, paths[0], paths[2], paths[1], paths[3], str(start[0]), str(start[1]),
                        str(end[0]), str(end[1])], capture_output=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(p.stderr.decode(errors="replace"))
    return p.stdout.decode("latin-1")
