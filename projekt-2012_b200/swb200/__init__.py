"""Python access to libswb200.so (the C ABI in include/swb200.h).

Used by the tests and bench.py.  The library is the product; this module only
marshals arguments.  Loading fails loudly when the shared library is missing:
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from collections.abc import Sequence as _Seq
from typing import List, Optional, Tuple

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "build", "libswb200.so")
CLI_PATH = os.path.join(PKG_DIR, "build", "SWalign")

SWB_OK = 0
SWB_EINVAL = 1
SWB_ENOMEM = 2
SWB_ENOMEM_BUDGET = 3
SWB_ETIMEOUT = 4
SWB_ECUDA = 5
SWB_EUNSUPPORTED = 6
SWB_EBUSY = 7
SWB_ENOTFOUND = 8

FLAG_TIE_ROWMAJOR = 0x1
FLAG_SCORE_ONLY = 0x2
FLAG_NO_SPECIAL = 0x4
FLAG_TEST_WITHHOLD = 0x80000000  # test hooks (include/swb200.h)
FLAG_TEST_PACK_ANY = 0x40000000


class Scoring(C.Structure):
    _fields_ = [("match", C.c_int32), ("mismatch", C.c_int32),
                ("gap_open", C.c_int32), ("gap_extend", C.c_int32)]


class XPoint(C.Structure):
    _fields_ = [("gap", C.c_int32), ("score", C.c_int32), ("row", C.c_int64), ("col", C.c_int64)]


class Result(C.Structure):
    _fields_ = [("score", C.c_int32),
                ("end_row", C.c_int64), ("end_col", C.c_int64),
                ("start_row", C.c_int64), ("start_col", C.c_int64),
                ("swapped", C.c_int32),
                ("rows", C.c_int64), ("cols", C.c_int64),
                ("stage1_ms", C.c_double), ("stage2_ms", C.c_double), ("total_ms", C.c_double),
                ("n_ops", C.c_int64), ("ops", C.c_void_p),
                ("n_xpoints", C.c_int64), ("xpoints", C.POINTER(XPoint)),
                ("xpoint_interval", C.c_int32), ("special_interval", C.c_int32),
                ("special_bytes", C.c_int64), ("kernel_launches", C.c_int32), ("host_bytes", C.c_int64)]


class PairRef(C.Structure):
    _fields_ = [("a_off", C.c_int64), ("a_len", C.c_int64), ("b_off", C.c_int64), ("b_len", C.c_int64)]


class BatchItem(C.Structure):
    _fields_ = [("score", C.c_int32), ("swapped", C.c_int32),
                ("end_row", C.c_int64), ("end_col", C.c_int64),
                ("start_row", C.c_int64), ("start_col", C.c_int64),
                ("ops_off", C.c_int64), ("n_ops", C.c_int64),
                ("xp_off", C.c_int64), ("n_xpoints", C.c_int64),
                ("traced", C.c_int32), ("xpoint_interval", C.c_int32)]


class BatchResult(C.Structure):
    _fields_ = [("npairs", C.c_int64), ("items", C.POINTER(BatchItem)),
                ("ops", C.c_void_p), ("ops_bytes", C.c_int64),
                ("xpoints", C.POINTER(XPoint)), ("n_xpoints", C.c_int64),
                ("n_traced", C.c_int64), ("cells", C.c_int64),
                ("stage1_ms", C.c_double), ("stage2_ms", C.c_double), ("total_ms", C.c_double),
                ("kernel_launches", C.c_int32)]


class ServerOptions(C.Structure):
    _fields_ = [("device", C.c_int32), ("hbm_budget_bytes", C.c_uint64), ("long_cells", C.c_int64),
                ("max_batch", C.c_int32), ("reserve_sms", C.c_int32), ("flags", C.c_uint32)]


class BlockBest(C.Structure):
    _fields_ = [("score", C.c_int32), ("row", C.c_int64), ("col", C.c_int64), ("key", C.c_uint64),
                ("stage1_ms", C.c_double)]


class RequestInfo(C.Structure):
    _fields_ = [("queued_ms", C.c_double), ("run_ms", C.c_double), ("total_ms", C.c_double),
                ("lane", C.c_int32), ("batch_size", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
                ("iterations", C.c_int64), ("max_batch_seen", C.c_int64), ("long_completed", C.c_int64),
                ("peak_reserved_bytes", C.c_uint64), ("cells_completed", C.c_int64)]


class Options(C.Structure):
    _fields_ = [("device", C.c_int32), ("hbm_budget_bytes", C.c_uint64),
                ("special_interval", C.c_int32), ("verbose", C.c_int32),
                ("cuda_stream", C.c_uint64), ("wait_limit_ms", C.c_uint32), ("host_spill_bytes", C.c_uint64)]


class SwbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"swb error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    """Loads libswb200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}` (no CPU fallback exists)")
        L = C.CDLL(LIB_PATH)
        L.swb_options_default.argtypes = [C.POINTER(Options)]
        L.swb_ctx_create.argtypes = [C.POINTER(Options), C.POINTER(C.c_void_p)]
        L.swb_ctx_create.restype = C.c_int
        L.swb_ctx_destroy.argtypes = [C.c_void_p]
        L.swb_last_error.argtypes = [C.c_void_p]
        L.swb_last_error.restype = C.c_char_p
        L.swb_scoring_parse.argtypes = [C.c_char_p] * 4 + [C.POINTER(Scoring)]
        L.swb_scoring_parse.restype = C.c_int
        L.swb_align_pair.argtypes = [C.c_void_p, C.c_char_p, C.c_int64, C.c_char_p, C.c_int64,
                                     C.POINTER(Scoring), C.c_uint32, C.POINTER(Result)]
        L.swb_align_pair.restype = C.c_int
        L.swb_align_pair_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                            C.POINTER(Scoring), C.c_uint32, C.POINTER(Result)]
        L.swb_align_pair_device.restype = C.c_int
        L.swb_score_block_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                                             C.c_void_p, C.c_int32, C.c_int64, C.c_int64, C.c_int64, C.c_int64,
                                             C.POINTER(Scoring), C.c_uint32, C.c_void_p, C.c_void_p,
                                             C.POINTER(BlockBest)]
        L.swb_score_block_device.restype = C.c_int
        L.swb_result_free.argtypes = [C.POINTER(Result)]
        L.swb_reference_geometry.argtypes = [C.c_int64, C.c_int64, C.POINTER(C.c_int32),
                                             C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                             C.POINTER(C.c_int64)]
        L.swb_reference_geometry.restype = C.c_int
        L.swb_special_row_copy.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                           C.POINTER(C.c_int64)]
        L.swb_special_row_copy.restype = C.c_int
        L.swb_version.restype = C.c_char_p
        L.swb_batch_align.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                                      C.POINTER(Scoring), C.c_uint32, C.c_double, C.POINTER(BatchResult)]
        L.swb_batch_align.restype = C.c_int
        L.swb_batch_align_device.argtypes = L.swb_batch_align.argtypes
        L.swb_batch_align_device.restype = C.c_int
        L.swb_batch_result_free.argtypes = [C.POINTER(BatchResult)]
        L.swb_server_options_default.argtypes = [C.POINTER(ServerOptions)]
        L.swb_server_create.argtypes = [C.POINTER(ServerOptions), C.POINTER(Scoring), C.POINTER(C.c_void_p)]
        L.swb_server_create.restype = C.c_int
        L.swb_server_submit.argtypes = [C.c_void_p, C.c_char_p, C.c_int64, C.c_char_p, C.c_int64,
                                        C.POINTER(C.c_uint64)]
        L.swb_server_submit.restype = C.c_int
        L.swb_server_wait.argtypes = [C.c_void_p, C.c_uint64, C.c_int64, C.POINTER(Result),
                                      C.POINTER(RequestInfo)]
        L.swb_server_wait.restype = C.c_int
        L.swb_server_stats_get.argtypes = [C.c_void_p, C.POINTER(ServerStats)]
        L.swb_server_stats_get.restype = C.c_int
        L.swb_server_last_error.argtypes = [C.c_void_p]
        L.swb_server_last_error.restype = C.c_char_p
        L.swb_server_destroy.argtypes = [C.c_void_p]
        L.swb_probe_cell_peak.argtypes = [C.c_int32] + [C.POINTER(C.c_double)] * 5
        L.swb_probe_cell_peak.restype = C.c_int
        L.swb_probe_latency.argtypes = [C.c_int32, C.POINTER(C.c_double), C.c_int32]
        L.swb_probe_latency.restype = C.c_int
        L.swb_gap_lists.argtypes = [C.POINTER(Result), C.c_void_p, C.c_int64, C.POINTER(C.c_int64), C.c_void_p,
                                    C.c_int64, C.POINTER(C.c_int64)]
        L.swb_gap_lists.restype = C.c_int
        L.swb_gap_lists_write.argtypes = [C.POINTER(Result), C.c_char_p, C.c_char_p]
        L.swb_gap_lists_write.restype = C.c_int
        L.swb_fasta_load.argtypes = [C.c_char_p, C.c_uint32, C.POINTER(C.POINTER(FastaRecord)),
                                     C.POINTER(C.c_int64)]
        L.swb_fasta_load.restype = C.c_int
        L.swb_fasta_free.argtypes = [C.POINTER(FastaRecord), C.c_int64]
        L.swb_fasta_free.restype = None
        _lib = L
    return _lib


def scoring(match, mismatch, gap_open, gap_extend) -> Scoring:
    return Scoring(match, mismatch, gap_open, gap_extend)


@dataclass
class Alignment:
    score: int
    end_row: int
    end_col: int
    start_row: int
    start_col: int
    swapped: bool
    rows: int
    cols: int
    stage1_ms: float
    stage2_ms: float
    total_ms: float
    ops: str = ""
    xpoints: "_Seq" = field(default_factory=list)  # (row, col, score, gap) tuples, built on access
    xpoint_interval: int = 0
    special_interval: int = 0
    special_bytes: int = 0
    kernel_launches: int = 0
    n_ops: int = 0
    host_bytes: int = 0      # of special_bytes, kept in pinned host memory


@dataclass
class Batch:
    """Result of a batched call: per-pair arrays in the order of the pairs
    argument, and the alignments / crosspoints of the traced pairs."""
    score: "object"            # numpy int32 [n]
    end_row: "object"          # numpy int64 [n]
    end_col: "object"
    start_row: "object"
    start_col: "object"
    swapped: "object"
    traced: "object"
    ops: List[str]             # "" for pairs that were not traced
    xpoints: "object"           # xpoints[i]: list of (row, col, score, gap); () if not traced
    xpoint_interval: "object"
    n_traced: int
    cells: int
    stage1_ms: float
    stage2_ms: float
    total_ms: float
    kernel_launches: int


def _convert_batch(r: BatchResult) -> Batch:
    import numpy as np
    n = r.npairs
    size = C.sizeof(BatchItem)
    ctype_dt = {C.c_int32: np.int32, C.c_int64: np.int64}
    dt = np.dtype({"names": [f for f, _ in BatchItem._fields_],
                   "formats": [ctype_dt[t] for _, t in BatchItem._fields_],
                   "offsets": [getattr(BatchItem, f).offset for f, _ in BatchItem._fields_], "itemsize": size})
    arr = np.frombuffer(C.string_at(r.items, n * size), dtype=dt) if n else np.zeros(0, dtype=dt)

    def col(name, dtype):
        return np.array(arr[name], dtype=dtype)
    score, swapped = col("score", np.int32), col("swapped", np.int32)
    traced, xpi = col("traced", np.int32), col("xpoint_interval", np.int32)
    ops_off, n_ops = col("ops_off", np.int64), col("n_ops", np.int64)
    xp_off, n_xp = col("xp_off", np.int64), col("n_xpoints", np.int64)
    allops = C.string_at(r.ops, r.ops_bytes).decode() if r.ops and r.ops_bytes > 0 else ""
    ops = [""] * n
    idx = np.flatnonzero(traced)
    for i, o, no in zip(idx.tolist(), ops_off[idx].tolist(), n_ops[idx].tolist()):
        ops[i] = allops[o:o + no]
    xps = _PairXpoints(_xpoint_array(r.xpoints, r.n_xpoints), xp_off, np.where(traced != 0, n_xp, 0))
    return Batch(score, col("end_row", np.int64), col("end_col", np.int64), col("start_row", np.int64),
                 col("start_col", np.int64), swapped.astype(bool), traced.astype(bool), ops, xps, xpi,
                 r.n_traced, r.cells, r.stage1_ms, r.stage2_ms, r.total_ms, r.kernel_launches)


def pair_refs(refs) -> "C.Array":
    """(n, 4) int64 array of (a_off, a_len, b_off, b_len) -> ctypes array of PairRef."""
    import numpy as np
    a = np.ascontiguousarray(refs, dtype=np.int64).reshape(-1, 4)
    arr = (PairRef * len(a))()
    if len(a):
        C.memmove(arr, a.ctypes.data, a.nbytes)
    return arr


def _xpoint_array(ptr, count: int):
    """The count XPoint records at ptr as a numpy structured array in (row, col,
    score, gap) field order (a copy; tolist() of a slice gives the tuples)."""
    import numpy as np
    size = C.sizeof(XPoint)
    dt = np.dtype({"names": ["row", "col", "score", "gap"], "formats": [np.int64, np.int64, np.int32, np.int32],
                   "offsets": [XPoint.row.offset, XPoint.col.offset, XPoint.score.offset, XPoint.gap.offset],
                   "itemsize": size})
    if count <= 0 or not ptr:
        return np.zeros(0, dtype=dt)
    return np.frombuffer(C.string_at(C.cast(ptr, C.c_void_p).value, count * size), dtype=dt)


class _PairXpoints:
    """Per-pair crosspoint lists of a batch, built on access: xp[i] is the list of
    (row, col, score, gap) tuples of pair i (() for pairs that were not traced).
    A batch with 1,000 traced pairs holds about 500,000 crosspoints; turning all
    of them into tuples up front took 100 ms per call."""

    def __init__(self, raw, off, cnt):
        self._raw, self._off, self._cnt = raw, off, cnt

    def __len__(self):
        return len(self._off)

    def __getitem__(self, i):
        n = int(self._cnt[i])
        if n <= 0:
            return ()
        o = int(self._off[i])
        return self._raw[o:o + n].tolist()

    def __iter__(self):
        return (self[i] for i in range(len(self)))

    def __eq__(self, other):
        return len(self) == len(other) and all(x == y for x, y in zip(self, other))


class _Xpoints(_Seq):
    """A pair's crosspoints, (row, col, score, gap) tuples built on first access:
    the records are copied to the host with the result, but 40,000 crosspoints
    (the 1 Mbp pair) took 10 ms to turn into tuples, time the GPU sat idle
    between alignments.  Compares equal to any sequence of the same tuples."""

    def __init__(self, arr):
        self._arr, self._list = arr, None

    def _tuples(self) -> list:
        if self._list is None:
            self._list = self._arr.tolist() if self._arr is not None else []
        return self._list

    def __len__(self):
        return len(self._arr) if self._arr is not None else 0

    def __getitem__(self, i):
        return self._tuples()[i]

    def __iter__(self):
        return iter(self._tuples())

    def __eq__(self, other):
        if isinstance(other, _Xpoints):
            other = other._tuples()
        return isinstance(other, _Seq) and self._tuples() == list(other)

    def __repr__(self):
        return repr(self._tuples())


def _convert(r: Result) -> Alignment:
    ops = C.string_at(r.ops, r.n_ops).decode() if r.n_ops > 0 and r.ops else ""
    xps = _Xpoints(_xpoint_array(r.xpoints, r.n_xpoints) if r.n_xpoints > 0 and r.xpoints else None)
    return Alignment(r.score, r.end_row, r.end_col, r.start_row, r.start_col, bool(r.swapped),
                     r.rows, r.cols, r.stage1_ms, r.stage2_ms, r.total_ms, ops, xps,
                     r.xpoint_interval, r.special_interval, r.special_bytes, r.kernel_launches,
                     r.n_ops, r.host_bytes)


FASTA_MULTI = 0x1
FASTA_UPPER = 0x2


class FastaRecord(C.Structure):
    _fields_ = [("name", C.c_char_p), ("seq", C.c_void_p), ("len", C.c_int64)]


def fasta_load(path: str, flags: int = 0) -> List[Tuple[str, bytes]]:
    """Records (name, sequence bytes) of a FASTA file: flags 0 = the reference
    loader's single-record rules (src/FASTA.cpp:39-86); FASTA_MULTI = every '>'
    line opens a record; FASTA_UPPER folds lower case."""
    recs, n = C.POINTER(FastaRecord)(), C.c_int64()
    rc = lib().swb_fasta_load(path.encode(), flags, C.byref(recs), C.byref(n))
    if rc != SWB_OK:
        raise SwbError(rc, lib().swb_last_error(None).decode())
    try:
        return [(recs[i].name.decode(errors="replace"), C.string_at(recs[i].seq, recs[i].len))
                for i in range(n.value)]
    finally:
        lib().swb_fasta_free(recs, n.value)


class Gap(C.Structure):
    _fields_ = [("begin", C.c_int32), ("length", C.c_int32)]


def _result_view(ops: str, start_row: int, start_col: int):
    """A Result carrying an operation string (kept alive by the returned buffer)."""
    raw = ops.encode()
    buf = C.create_string_buffer(raw, len(raw) + 1)
    r = Result()
    r.ops = C.cast(buf, C.c_void_p)
    r.n_ops = len(raw)
    r.start_row = start_row
    r.start_col = start_col
    return r, buf


def gap_lists(al) -> Tuple[List[Tuple[int, int]], List[Tuple[int, int]]]:
    """The alignment's gap lists in the reference renderer's format
    (src/Visualisation.cpp:11-127): for the first (rows) and second (columns)
    sequence, (begin, length) = `length` gaps before the base at index `begin`.
    `al` needs ops, start_row and start_col (an Alignment)."""
    r, keep = _result_view(al.ops, al.start_row, al.start_col)
    n1, n2 = C.c_int64(), C.c_int64()
    rc = lib().swb_gap_lists(C.byref(r), None, 0, C.byref(n1), None, 0, C.byref(n2))
    if rc != SWB_OK and (n1.value == 0 and n2.value == 0):
        raise SwbError(rc, lib().swb_last_error(None).decode())
    a, b = (Gap * max(1, n1.value))(), (Gap * max(1, n2.value))()
    rc = lib().swb_gap_lists(C.byref(r), C.cast(a, C.c_void_p), n1.value, C.byref(n1), C.cast(b, C.c_void_p),
                             n2.value, C.byref(n2))
    if rc != SWB_OK:
        raise SwbError(rc, lib().swb_last_error(None).decode())
    del keep
    return ([(a[i].begin, a[i].length) for i in range(n1.value)],
            [(b[i].begin, b[i].length) for i in range(n2.value)])


def write_gap_lists(al, first_path: str, second_path: str) -> None:
    """Writes the two gap lists as the reference's binary files (int32 begin,
    int32 length records)."""
    r, keep = _result_view(al.ops, al.start_row, al.start_col)
    rc = lib().swb_gap_lists_write(C.byref(r), first_path.encode(), second_path.encode())
    del keep
    if rc != SWB_OK:
        raise SwbError(rc, lib().swb_last_error(None).decode())


class Context:
    """One device context (owns a CUDA stream and reusable device buffers)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, special_interval: int = 0,
                 cuda_stream: int = 0, verbose: int = 0, wait_limit_ms: int = 0, host_spill_bytes: int = 0):
        L = lib()
        o = Options()
        L.swb_options_default(C.byref(o))
        o.device = device
        o.hbm_budget_bytes = hbm_budget_bytes
        o.special_interval = special_interval
        o.cuda_stream = cuda_stream
        o.verbose = verbose
        o.wait_limit_ms = wait_limit_ms
        o.host_spill_bytes = host_spill_bytes
        h = C.c_void_p()
        rc = L.swb_ctx_create(C.byref(o), C.byref(h))
        if rc != SWB_OK:
            raise SwbError(rc, L.swb_last_error(None).decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().swb_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _err(self, rc):
        raise SwbError(rc, lib().swb_last_error(self._h).decode())

    def align(self, a: bytes, b: bytes, sc: Scoring, flags: int = 0) -> Alignment:
        r = Result()
        rc = lib().swb_align_pair(self._h, a, len(a), b, len(b), C.byref(sc), flags, C.byref(r))
        if rc != SWB_OK:
            self._err(rc)
        try:
            return _convert(r)
        finally:
            lib().swb_result_free(C.byref(r))

    def align_ptr(self, p_a: int, la: int, p_b: int, lb: int, sc: Scoring, flags: int = 0) -> Alignment:
        """Host sequences given by address (e.g. pinned buffers)."""
        r = Result()
        fn = lib().swb_align_pair
        rc = fn(self._h, C.cast(C.c_void_p(p_a), C.c_char_p), la, C.cast(C.c_void_p(p_b), C.c_char_p), lb,
                C.byref(sc), flags, C.byref(r))
        if rc != SWB_OK:
            self._err(rc)
        try:
            return _convert(r)
        finally:
            lib().swb_result_free(C.byref(r))

    def align_device(self, d_rows: int, rows: int, d_cols: int, cols: int, sc: Scoring,
                     flags: int = 0) -> Alignment:
        r = Result()
        rc = lib().swb_align_pair_device(self._h, C.c_void_p(d_rows), rows, C.c_void_p(d_cols), cols,
                                         C.byref(sc), flags, C.byref(r))
        if rc != SWB_OK:
            self._err(rc)
        try:
            return _convert(r)
        finally:
            lib().swb_result_free(C.byref(r))

    def batch_align(self, seq, refs, sc: Scoring, flags: int = 0, trace_frac: float = 0.0,
                    seq_ptr: Optional[int] = None, device: bool = False) -> Batch:
        """Aligns the pairs refs[i] = (a_off, a_len, b_off, b_len) of the buffer seq
        (bytes / numpy uint8), or of the buffer at address seq_ptr (host memory, or
        device memory when device=True, len(seq) bytes when seq is an int)."""
        import numpy as np
        pr = pair_refs(refs)
        if seq_ptr is None:
            buf = np.frombuffer(seq, dtype=np.uint8) if isinstance(seq, (bytes, bytearray)) else \
                np.ascontiguousarray(seq, dtype=np.uint8)
            ptr, nbytes = buf.ctypes.data, buf.nbytes
        else:
            ptr, nbytes = seq_ptr, int(seq)
        r = BatchResult()
        fn = lib().swb_batch_align_device if device else lib().swb_batch_align
        rc = fn(self._h, C.c_void_p(ptr), nbytes, pr, len(pr), C.byref(sc), flags, trace_frac, C.byref(r))
        if rc != SWB_OK:
            self._err(rc)
        try:
            return _convert_batch(r)
        finally:
            lib().swb_batch_result_free(C.byref(r))

    def trace(self):
        """Stage-1 strip trace of the last call: numpy array [strips, 3] of
        (start ns, end ns, SM id); needs Context(verbose=2)."""
        import numpy as np
        cnt = C.c_int64(0)
        fn = lib().swb_trace_copy
        fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int64)]
        fn(self._h, None, 0, C.byref(cnt)) if False else None
        probe = np.zeros(3, dtype=np.int64)
        fn(self._h, probe.ctypes.data, 0, C.byref(cnt))
        out = np.zeros((cnt.value, 3), dtype=np.int64)
        rc = fn(self._h, out.ctypes.data, 3 * cnt.value, C.byref(cnt))
        if rc != SWB_OK:
            self._err(rc)
        return out

    def special_row(self, idx: int, cols: int):
        import numpy as np
        out = np.zeros((cols, 2), dtype=np.int32)
        interval = C.c_int64(0)
        rc = lib().swb_special_row_copy(self._h, idx, out.ctypes.data, cols, C.byref(interval))
        if rc != SWB_OK:
            self._err(rc)
        return out, interval.value


def reference_geometry(rows: int, cols: int):
    G, T = C.c_int32(), C.c_int32()
    P1, P2 = C.c_int64(), C.c_int64()
    rc = lib().swb_reference_geometry(rows, cols, C.byref(G), C.byref(T), C.byref(P1), C.byref(P2))
    return rc, G.value, T.value, P1.value, P2.value


def version() -> str:
    return lib().swb_version().decode()


def probe_cell_peak(device: int = 0) -> dict:
    """Measured peak cell-update rate of the stage-1 per-cell instruction mix
    (swb_probe_cell_peak) and single-op rates."""
    v = [C.c_double() for _ in range(5)]
    rc = lib().swb_probe_cell_peak(device, *[C.byref(x) for x in v])
    if rc != SWB_OK:
        raise SwbError(rc, "probe failed")
    return {"cells_per_s": v[0].value, "iadd_per_s": v[1].value, "viaddmax_per_s": v[2].value,
            "vimax3_per_s": v[3].value, "probe_ms": v[4].value}


def probe_latency(device: int = 0) -> dict:
    """Dependent-chain latency in SM cycles per op (swb_probe_latency)."""
    v = (C.c_double * 6)()
    rc = lib().swb_probe_latency(device, v, 6)
    if rc != SWB_OK:
        raise SwbError(rc, "latency probe failed")
    names = ["iadd", "max_add_c", "viaddmax", "vimax3", "viaddmax_relu", "max_c"]
    return dict(zip(names, list(v)))


class Server:
    """The serving loop (swb_server_*): submit requests at any time, wait for
    each one's result; short requests are batched per iteration, long ones run
    in a second lane beside them."""

    def __init__(self, sc: Scoring, device: int = 0, hbm_budget_bytes: int = 0, long_cells: int = 0,
                 max_batch: int = 0, reserve_sms: int = 0, flags: int = 0):
        L = lib()
        o = ServerOptions()
        L.swb_server_options_default(C.byref(o))
        o.device, o.hbm_budget_bytes, o.long_cells = device, hbm_budget_bytes, long_cells
        o.max_batch, o.reserve_sms, o.flags = max_batch, reserve_sms, flags
        h = C.c_void_p()
        self._sc = Scoring(sc.match, sc.mismatch, sc.gap_open, sc.gap_extend)
        rc = L.swb_server_create(C.byref(o), C.byref(self._sc), C.byref(h))
        if rc != SWB_OK:
            raise SwbError(rc, L.swb_last_error(None).decode())
        self._h = h

    def submit(self, a: bytes, b: bytes) -> int:
        rid = C.c_uint64(0)
        rc = lib().swb_server_submit(self._h, a, len(a), b, len(b), C.byref(rid))
        if rc != SWB_OK:
            raise SwbError(rc, lib().swb_last_error(None).decode())
        return rid.value

    def wait(self, rid: int, timeout_ms: int = -1):
        """(Alignment, info dict) or None when timeout_ms ran out."""
        r, info = Result(), RequestInfo()
        L = lib()
        rc = L.swb_server_wait(self._h, rid, timeout_ms, C.byref(r), C.byref(info))
        if rc == SWB_ETIMEOUT:
            return None
        if rc != SWB_OK:
            raise SwbError(rc, (L.swb_server_last_error(self._h) or b"").decode())
        try:
            return _convert(r), {"queued_ms": info.queued_ms, "run_ms": info.run_ms, "total_ms": info.total_ms,
                                 "lane": info.lane, "batch_size": info.batch_size}
        finally:
            L.swb_result_free(C.byref(r))

    def stats(self) -> dict:
        st = ServerStats()
        lib().swb_server_stats_get(self._h, C.byref(st))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib().swb_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
