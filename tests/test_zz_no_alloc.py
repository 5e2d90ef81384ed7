"""swb_score_pair_noalloc: the entry point for callers that cannot allocate
device memory (code inside another framework's memory pool or under a
no-allocation policy).  Its scratch is a fixed array inside the library; this
checks it gives exactly the same score and end cell as swb_align_pair_device on
two calls in a row (the second call runs on scratch the first one left behind),
and that sizes beyond the fixed limits are refused before any GPU work.

Kept in a file of its own that pytest collects last."""
import ctypes as C
import random

import pytest

import swb200

pytestmark = pytest.mark.gpu


class Score(C.Structure):
    _fields_ = [("score", C.c_int32), ("end_row", C.c_int64), ("end_col", C.c_int64)]


def _noalloc():
    L = swb200.lib()
    fn = L.swb_score_pair_noalloc
    fn.argtypes = [C.c_int32, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64,
                   C.POINTER(swb200.Scoring), C.c_uint32, C.c_uint64, C.POINTER(Score)]
    fn.restype = C.c_int
    L.swb_noalloc_last_error.restype = C.c_char_p
    return fn, L.swb_noalloc_last_error


def _pair(seed, m, frac):
    rng = random.Random(seed)
    a = bytes(rng.choice(b"ACGT") for _ in range(m))
    st = rng.randint(0, m // 4)
    core = bytearray(a[st:st + int(m * frac)])
    for i in range(len(core)):
        if rng.random() < 0.06:
            core[i] = rng.choice(b"ACGT")
    b = bytes(rng.choice(b"ACGT") for _ in range(500)) + bytes(core)
    return (a, b) if len(a) >= len(b) else (b, a)


def test_noalloc_matches_existing_entry_point_on_two_calls_in_a_row():
    import torch
    fn, err = _noalloc()
    sc = swb200.scoring(1, -3, -5, -2)
    pairs = [_pair(1, 30000, 0.5), _pair(2, 7000, 0.3)]
    tensors = [(torch.frombuffer(bytearray(r), dtype=torch.uint8).cuda(),
                torch.frombuffer(bytearray(c), dtype=torch.uint8).cuda()) for r, c in pairs]
    stream = torch.cuda.current_stream().cuda_stream
    got = []
    for (r, c), (tr, tc) in zip(pairs, tensors):          # two calls in a row
        out = Score()
        rc = fn(0, tr.data_ptr(), len(r), tc.data_ptr(), len(c), C.byref(sc), 0, stream, C.byref(out))
        assert rc == swb200.SWB_OK, err()
        got.append((out.score, out.end_row, out.end_col))
    with swb200.Context(device=0) as ctx:
        for (r, c), (tr, tc), g in zip(pairs, tensors, got):
            ref = ctx.align_device(tr.data_ptr(), len(r), tc.data_ptr(), len(c), sc, swb200.FLAG_SCORE_ONLY)
            assert g == (ref.score, ref.end_row, ref.end_col)
            assert g[0] > 0


def test_noalloc_refuses_sizes_beyond_its_scratch():
    fn, err = _noalloc()
    sc = swb200.scoring(1, -3, -5, -2)
    out = Score()
    too_many_cols = (1 << 20) + 1
    rc = fn(0, C.c_void_p(1), too_many_cols, C.c_void_p(1), too_many_cols, C.byref(sc), 0, 0, C.byref(out))
    assert rc == swb200.SWB_EUNSUPPORTED
    assert b"SWB_NOALLOC_MAX" in err()


def _compare_with_pair_path(pairs, flags=0):
    import torch
    fn, err = _noalloc()
    sc = swb200.scoring(1, -3, -5, -2)
    stream = torch.cuda.current_stream().cuda_stream
    with swb200.Context(device=0) as ctx:
        for r, c in pairs:
            tr = torch.frombuffer(bytearray(r), dtype=torch.uint8).cuda()
            tc = torch.frombuffer(bytearray(c), dtype=torch.uint8).cuda()
            out = Score()
            rc = fn(0, tr.data_ptr(), len(r), tc.data_ptr(), len(c), C.byref(sc), flags, stream, C.byref(out))
            assert rc == swb200.SWB_OK, err()
            ref = ctx.align_device(tr.data_ptr(), len(r), tc.data_ptr(), len(c), sc,
                                   swb200.FLAG_SCORE_ONLY | flags)
            assert (out.score, out.end_row, out.end_col) == (ref.score, ref.end_row, ref.end_col), (len(r), len(c))


def test_noalloc_at_its_limits_and_with_the_rowmajor_tie():
    """More strips than the scratch holds warps for (the grid is capped), the
    widest pair the hand-off row allows (cols = SWB_NOALLOC_MAX_COLS), and the
    row-major tie rule on a pair of all-equal maxima."""
    rng = random.Random(11)
    tall = bytes(rng.choice(b"ACGT") for _ in range(2_200_000))
    tall_cols = tall[1_000_000:1_000_700]
    wide = bytes(rng.choice(b"ACGT") for _ in range(1 << 20))
    wide_cols = bytes(c if rng.random() > 0.05 else rng.choice(b"ACGT") for c in wide)
    _compare_with_pair_path([(tall, tall_cols), (wide, wide_cols)])
    _compare_with_pair_path([(b"A" * 3000, b"A" * 900)], swb200.FLAG_TIE_ROWMAJOR)


def test_noalloc_set_up_call_with_empty_pair():
    """rows = cols = 0 does only the per-device set-up and scores 0 at (0, 0)."""
    fn, err = _noalloc()
    sc = swb200.scoring(1, -3, -5, -2)
    out = Score()
    out.score = -1
    rc = fn(0, None, 0, None, 0, C.byref(sc), 0, 0, C.byref(out))
    assert rc == swb200.SWB_OK, err()
    assert (out.score, out.end_row, out.end_col) == (0, 0, 0)


def test_noalloc_refuses_a_capturing_stream_and_keeps_the_capture():
    """On a stream that is capturing a graph the call returns SWB_EINVAL without
    touching the stream; the capture ends normally and its graph replays."""
    import torch
    fn, err = _noalloc()
    sc = swb200.scoring(1, -3, -5, -2)
    r, c = _pair(5, 3000, 0.5)
    tr = torch.frombuffer(bytearray(r), dtype=torch.uint8).cuda()
    tc = torch.frombuffer(bytearray(c), dtype=torch.uint8).cuda()
    x = torch.zeros(16, device="cuda")
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    rcs = []
    with torch.cuda.graph(g, stream=s):
        x.add_(1)
        out = Score()
        rcs.append(fn(0, tr.data_ptr(), len(r), tc.data_ptr(), len(c), C.byref(sc), 0, s.cuda_stream,
                      C.byref(out)))
    assert rcs == [swb200.SWB_EINVAL], err()
    assert b"capturing" in err()
    g.replay()
    torch.cuda.synchronize()
    assert float(x[0]) == 1.0
    out = Score()   # outside the capture the same call works
    assert fn(0, tr.data_ptr(), len(r), tc.data_ptr(), len(c), C.byref(sc), 0, s.cuda_stream, C.byref(out)) == 0
    assert out.score > 0
