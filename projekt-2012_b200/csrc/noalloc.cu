// noalloc.cu -- stage-1 scoring for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at all: code that runs inside another
// framework's memory pool or under a no-allocation policy on the device, a
// plugin whose host process forbids new device allocations once it is up, or a
// caller that wants the whole call to be free of allocation so it cannot fail
// on memory.  swb_score_pair_noalloc() serves them: the caller passes the two
// sequences (device memory) and a host result struct, and every piece of
// scratch the stage-1 kernel needs lives in one file-scope device array,
// g_noalloc_scratch, of fixed size (kNoAllocScratchBytes, about 16.1 MiB), which
// every GPU that loads this library holds until the process exits.
//
// The array's name is only a host-side stand-in in host code; the device address
// is looked up once per device with cudaGetSymbolAddress (with that device
// current) on the first call on the device, and handed to the kernel.  That
// first call therefore does the set-up and should come before any stream
// capture.  All calls share the one array, which keeps the last call's contents:
// the row buffer's tags and the error flags are reset at the start of every call.
// Each device has its own copy of the array, so calls on different devices are
// independent; calls on the same device that overlap on the GPU (from two
// streams or two host threads) race on it and must be serialised by the caller.
#include <algorithm>
#include <cstdio>
#include <mutex>

#include "swb_internal.h"

namespace swb {
namespace {

constexpr int64_t kMaxCols = SWB_NOALLOC_MAX_COLS;
constexpr int64_t kMaxRows = SWB_NOALLOC_MAX_ROWS;
constexpr int64_t kMaxWarps = 4096;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffHbuf = 0;
constexpr size_t kOffWbest = kOffHbuf + align256(sizeof(int4) * (size_t)kMaxCols);
constexpr size_t kOffBest = kOffWbest + align256(sizeof(BestRec) * (size_t)kMaxWarps);
constexpr size_t kOffErr = kOffBest + align256(sizeof(BestRec));
constexpr size_t kNoAllocScratchBytes = kOffErr + align256(4 * sizeof(int32_t));

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void *g_scratch_addr[kMaxDevices] = {nullptr};

thread_local char g_err[256];

int noalloc_fail(int code, const char *msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return code;
}

}  // namespace
}  // namespace swb

extern "C" const char *swb_noalloc_last_error(void) { return swb::g_err; }

extern "C" int swb_score_pair_noalloc(int32_t device, const void *d_rows, int64_t rows, const void *d_cols,
                                      int64_t cols, const swb_scoring *sc, uint32_t flags, uint64_t cuda_stream,
                                      swb_score *out) {
    using namespace swb;
    if (!out || !sc || rows < 0 || cols < 0 || rows < cols || (rows > 0 && !d_rows) || (cols > 0 && !d_cols))
        return noalloc_fail(SWB_EINVAL, "swb_score_pair_noalloc: bad arguments (rows >= cols required)");
    if (sc->match < 1 || sc->mismatch > -1 || sc->gap_open > -1 || sc->gap_extend > -1)
        return noalloc_fail(SWB_EINVAL, "One or more scoring values were not usable!");
    if (cols > kMaxCols || rows > kMaxRows)
        return noalloc_fail(SWB_EUNSUPPORTED,
                            "swb_score_pair_noalloc: sequence longer than the fixed scratch allows "
                            "(rows <= SWB_NOALLOC_MAX_ROWS, cols <= SWB_NOALLOC_MAX_COLS)");
    const long double worst = (long double)std::max(std::max(sc->match, -sc->mismatch),
                                                    std::max(-sc->gap_open, -sc->gap_extend)) *
                              (long double)(rows + cols + 2);
    if (worst > 2.0e9L) return noalloc_fail(SWB_EUNSUPPORTED, "scores would leave the int32 range");
    if (device < 0 || device >= kMaxDevices) return noalloc_fail(SWB_EINVAL, "device ordinal out of range");
    out->score = 0;
    out->end_row = 0;
    out->end_col = 0;

    int prev = -1;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return noalloc_fail(SWB_ECUDA, cudaGetErrorString(e));
    struct Restore {
        int d;
        ~Restore() {
            if (d >= 0) cudaSetDevice(d);
        }
    } restore{prev};

    // the call copies its result to the host and waits, which a stream capture
    // cannot record: refuse it on a capturing stream rather than break the capture
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        const cudaError_t ce = cudaStreamIsCapturing((cudaStream_t)(uintptr_t)cuda_stream, &cs);
        if (ce != cudaSuccess || cs != cudaStreamCaptureStatusNone)
            return noalloc_fail(SWB_EINVAL, "swb_score_pair_noalloc: the stream is capturing a graph");
    }

    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        if (!g_scratch_addr[device]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) return noalloc_fail(SWB_ECUDA, cudaGetErrorString(e));
            g_scratch_addr[device] = p;
        }
        base = (unsigned char *)g_scratch_addr[device];
    }
    // an empty pair scores 0 at (0, 0); such a call does only the set-up above
    if (rows == 0 || cols == 0) return SWB_OK;
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
        return noalloc_fail(SWB_ECUDA, cudaGetErrorString(e));
    Stage1Plan plan = stage1_plan(rows, cols, sms, 16, false);
    if ((int64_t)plan.blocks * plan.warps_per_block > kMaxWarps) plan.blocks = (int)(kMaxWarps / plan.warps_per_block);

    Stage1Args a{};
    a.rows = (const uint8_t *)d_rows;
    a.cols = (const uint8_t *)d_cols;
    a.m = rows;
    a.n = cols;
    a.open = sc->gap_open;
    a.ext = sc->gap_extend;
    a.gx = std::max(sc->gap_open, sc->gap_extend);
    a.mt1 = sc->match - sc->gap_open;
    a.mm1 = sc->mismatch - sc->gap_open;
    a.hbuf = (int4 *)(base + kOffHbuf);
    a.wbest = (BestRec *)(base + kOffWbest);
    a.best = (BestRec *)(base + kOffBest);
    a.err = (int32_t *)(base + kOffErr);
    a.gbest = a.err + 2;
    a.srows = nullptr;
    a.sr_every = 1;
    a.nsr = 0;
    a.nstrips = plan.nstrips;
    int32_t G = 0, T = 0;
    int64_t P1 = 0, P2 = 0;
    const bool refok = reference_geometry(rows, cols, &G, &T, &P1, &P2);
    a.tie.mode = ((flags & SWB_FLAG_TIE_ROWMAJOR) || !refok) ? kTieRowMajor : kTieReference;
    a.tie.G = G;
    a.tie.T = T;
    a.tie.C = refok ? P2 / G : 1;

    cudaStream_t st = (cudaStream_t)(uintptr_t)cuda_stream;
    BestRec best{};
    int32_t errh[2] = {0, 0};
    if ((e = cudaMemsetAsync(a.hbuf, 0xFF, sizeof(int4) * (size_t)cols, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(a.err, 0, 4 * sizeof(int32_t), st)) != cudaSuccess ||
        (e = stage1_launch(a, plan, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&best, a.best, sizeof best, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(errh, a.err, sizeof errh, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return noalloc_fail(SWB_ECUDA, cudaGetErrorString(e));
    if (errh[0] != 0) return noalloc_fail(SWB_ETIMEOUT, "stage 1: a bounded wait between strips ran out");
    if (best.valid) {
        out->score = best.ho - sc->gap_open;
        out->end_row = best.row;
        out->end_col = best.col;
    }
    return SWB_OK;
}
