// api.cpp -- context, device buffers and the pair entry points of libswb200.so.
//
// Host orchestration that replaces src/main.cu:102-249 (load -> device ->
// stage 1 -> reduction -> stage 2) without any process exit, file I/O or
// per-step host round trips: the whole of stage 1 is one persistent launch and
// the special rows stay in HBM (the reference appends them to temp/row_<R>
// files, src/Builders.cpp:41-61).
#include <algorithm>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ctx.h"
#include "batch.h"
#include "traceback.h"

#define SWB_VERSION_STRING "swb200 0.1.0 (sm_100a)"

namespace {
thread_local std::string g_thread_err;
}  // namespace

namespace swb {

double trace_now_ms() {
    static const auto t0 = std::chrono::steady_clock::now();
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

bool trace_on() {
    static const bool on = std::getenv("SWB_SERVE_TRACE") != nullptr;
    return on;
}

cudaError_t DevBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    const double t0 = trace_on() ? trace_now_ms() : 0.0;
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    cap = 0;
    size_t want = bytes < 256 ? 256 : bytes;
    cudaError_t e = cudaMallocAsync(&p, want, st);
    if (e == cudaSuccess) cap = want;
    else p = nullptr;
    if (trace_on() && want >= (64u << 20))
        std::fprintf(stderr, "swb trace %.1f grow %.1f MB in %.2f ms\n", t0, want / 1e6, trace_now_ms() - t0);
    return e;
}

void DevBuf::release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    cap = 0;
}

cudaError_t HostBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    size_t want = bytes < 4096 ? 4096 : bytes;
    cudaError_t e = cudaMallocHost(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
}

void HostBuf::release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
}

cudaError_t MappedBuf::ensure(size_t bytes) {
    if (bytes <= cap && p) return cudaSuccess;
    release();
    cudaError_t e = cudaHostAlloc(&p, bytes < 256 ? 256 : bytes, cudaHostAllocMapped | cudaHostAllocPortable);
    if (e != cudaSuccess) {
        p = nullptr;
        return e;
    }
    if ((e = cudaHostGetDevicePointer(&dp, p, 0)) != cudaSuccess) {
        release();
        return e;
    }
    cap = bytes < 256 ? 256 : bytes;
    return cudaSuccess;
}

void MappedBuf::release() {
    if (p) cudaFreeHost(p);
    p = dp = nullptr;
    cap = 0;
}

int ctx_fail(swb_ctx *ctx, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf;
    g_thread_err = buf;
    return code;
}

int ctx_cuda_fail(swb_ctx *ctx, cudaError_t e, const char *what) {
    return ctx_fail(ctx, SWB_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

cudaError_t ctx_get(swb_ctx *c, void *dst, const void *dev_src, size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    cudaError_t e;
    if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess || (e = c->h_io.ensure(bytes)) != cudaSuccess ||
        (e = cudaMemcpyAsync(c->h_io.p, dev_src, bytes, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c->stream)) != cudaSuccess)
        return e;
    std::memcpy(dst, c->h_io.p, bytes);
    return cudaSuccess;
}

cudaError_t ctx_put(swb_ctx *c, void *dev_dst, const void *src, size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    cudaError_t e;
    if ((e = cudaStreamSynchronize(c->stream)) != cudaSuccess || (e = c->h_io.ensure(bytes)) != cudaSuccess)
        return e;
    std::memcpy(c->h_io.p, src, bytes);
    return cudaMemcpyAsync(dev_dst, c->h_io.p, bytes, cudaMemcpyHostToDevice, c->stream);
}

}  // namespace swb

using swb::ctx_fail;
using swb::ctx_cuda_fail;
using swb::DevBuf;

namespace swb {

static int64_t pad_len(int64_t len, int64_t parts) {
    if (len <= 0 || parts <= 0) return len;
    const int64_t C = (len + parts - 1) / parts;
    if (len % C == 0) return len;
    return len + (C - len % C);
}

bool reference_geometry(int64_t rows, int64_t cols, int32_t *G, int32_t *T, int64_t *P1, int64_t *P2) {
    int32_t blocks = 2, threads = 5;
    if ((int64_t)threads * blocks * 2 > cols) blocks = (int32_t)((float)cols / (float)(threads * 2));
    if (blocks == 0) {
        blocks = 1;
        threads = (int32_t)(cols / 4);
    }
    *G = blocks;
    *T = threads;
    *P1 = pad_len(rows, 4);
    *P2 = pad_len(cols, blocks);
    return threads > 0;
}

}  // namespace swb

extern "C" {

void swb_options_default(swb_options *o) {
    std::memset(o, 0, sizeof *o);
    o->device = 0;
    o->hbm_budget_bytes = 0;
    o->special_interval = 0;
    o->verbose = 0;
    o->cuda_stream = 0;
}

int swb_ctx_create(const swb_options *opts, swb_ctx **out) {
    if (!out) return ctx_fail(nullptr, SWB_EINVAL, "swb_ctx_create: out is NULL");
    *out = nullptr;
    swb_ctx *c = new (std::nothrow) swb_ctx();
    if (!c) return ctx_fail(nullptr, SWB_ENOMEM, "swb_ctx_create: out of host memory");
    if (opts) c->opts = *opts;
    else swb_options_default(&c->opts);
    if (c->opts.hbm_budget_bytes == 0) c->opts.hbm_budget_bytes = 64ULL << 30;
    c->device = c->opts.device;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= 0) {
        delete c;
        return ctx_fail(nullptr, SWB_ECUDA, "no CUDA device: %s", cudaGetErrorString(e));
    }
    if (c->device < 0 || c->device >= ndev) {
        const int dev = c->device;
        delete c;
        return ctx_fail(nullptr, SWB_EINVAL, "device %d out of range (%d devices)", dev, ndev);
    }
    if ((e = cudaSetDevice(c->device)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device)) != cudaSuccess ||
        (c->opts.cuda_stream == 0 &&
         (e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) ||
        (e = cudaEventCreate(&c->ev0)) != cudaSuccess || (e = cudaEventCreate(&c->ev1)) != cudaSuccess ||
        (e = cudaEventCreate(&c->ev2)) != cudaSuccess ||
        (e = swb::stage1_configure()) != cudaSuccess || (e = swb::batch_configure()) != cudaSuccess ||
        (e = swb::batch16_configure()) != cudaSuccess ||
        (e = swb::tb::walker_configure()) != cudaSuccess) {
        int rc = ctx_cuda_fail(nullptr, e, "swb_ctx_create");
        // release what was created before the failure
        if (c->ev0) cudaEventDestroy(c->ev0);
        if (c->ev1) cudaEventDestroy(c->ev1);
        if (c->ev2) cudaEventDestroy(c->ev2);
        if (c->stream && c->opts.cuda_stream == 0) cudaStreamDestroy(c->stream);
        delete c;
        return rc;
    }
    if (c->opts.cuda_stream != 0) {
        c->stream = (cudaStream_t)(uintptr_t)c->opts.cuda_stream;
        c->own_stream = false;
    }
    if (c->opts.wait_limit_ms > 0) {
        int khz = 0;  // the kernels bound their waits with clock64(), in SM cycles
        if (cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, c->device) != cudaSuccess || khz <= 0) khz = 2000000;
        c->wait_cycles = (int64_t)c->opts.wait_limit_ms * khz;
    }
    c->each_buf([c](DevBuf &b) { b.st = c->stream; });
    *out = c;
    return SWB_OK;
}

void swb_ctx_destroy(swb_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->each_buf([](DevBuf &b) { b.release(); });
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->h_stage.release();
    c->h_io.release();
    c->srows_h.release();
    c->scols_h.release();
    c->h_gin.release();
    c->h_gout.release();
    for (auto &g : c->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.graph) cudaGraphDestroy(g.graph);
    }
    if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->ev2) cudaEventDestroy(c->ev2);
    if (c->stream && c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char *swb_last_error(const swb_ctx *c) { return c ? c->err.c_str() : g_thread_err.c_str(); }

const char *swb_version(void) { return SWB_VERSION_STRING; }

int swb_scoring_parse(const char *match, const char *mismatch, const char *gap_open, const char *gap_extend,
                      swb_scoring *out) {
    if (!match || !mismatch || !gap_open || !gap_extend || !out)
        return ctx_fail(nullptr, SWB_EINVAL, "swb_scoring_parse: NULL argument");
    swb_scoring s;
    s.match = std::atoi(match);
    s.mismatch = std::atoi(mismatch);
    s.gap_open = std::atoi(gap_open);
    s.gap_extend = std::atoi(gap_extend);
    if (s.match < 1 || s.mismatch > -1 || s.gap_open > -1 || s.gap_extend > -1)
        return ctx_fail(nullptr, SWB_EINVAL, "One or more scoring values were not usable!");
    *out = s;
    return SWB_OK;
}

int swb_reference_geometry(int64_t rows, int64_t cols, int32_t *G, int32_t *T, int64_t *P1, int64_t *P2) {
    int32_t g = 0, t = 0;
    int64_t p1 = 0, p2 = 0;
    const bool ok = swb::reference_geometry(rows, cols, &g, &t, &p1, &p2);
    if (G) *G = g;
    if (T) *T = t;
    if (P1) *P1 = p1;
    if (P2) *P2 = p2;
    return ok ? SWB_OK : SWB_EUNSUPPORTED;
}

void swb_result_free(swb_result *r) {
    if (!r) return;
    std::free(r->ops);
    std::free(r->xpoints);
    r->ops = nullptr;
    r->xpoints = nullptr;
    r->n_ops = 0;
    r->n_xpoints = 0;
}

}  // extern "C"

namespace {

// Scoring values must stay in the exact int32 range of the recurrence for the
// lengths involved (|score| <= max(|s|) * (rows + cols)).
int check_scoring(swb_ctx *c, const swb_scoring *sc, int64_t rows, int64_t cols) {
    if (!sc) return ctx_fail(c, SWB_EINVAL, "scoring is NULL");
    if (sc->match < 1 || sc->mismatch > -1 || sc->gap_open > -1 || sc->gap_extend > -1)
        return ctx_fail(c, SWB_EINVAL, "One or more scoring values were not usable!");
    const long double worst = (long double)std::max<int64_t>(
                                  {(int64_t)sc->match, -(int64_t)sc->mismatch, -(int64_t)sc->gap_open,
                                   -(int64_t)sc->gap_extend}) *
                              (long double)(rows + cols + 2);
    if (worst > 2.0e9L) return ctx_fail(c, SWB_EUNSUPPORTED, "scores would leave the int32 range");
    return SWB_OK;
}

// Runs stage 1 on device sequences already in the context's buffers.

// One block of a pair split into blocks (swb_score_block_device): boundaries in,
// boundaries out, tie keys over the whole matrix.
struct BlockIo {
    const int2 *top = nullptr, *left = nullptr;
    int32_t corner = 0;
    int64_t r0 = 0, c0 = 0, full_m = 0, full_n = 0;
    int2 *bottom = nullptr, *right = nullptr;
};

int run_stage1(swb_ctx *c, const uint8_t *d_rows, int64_t m, const uint8_t *d_cols, int64_t n,
               const swb_scoring *sc, uint32_t flags, int64_t sr_interval_rows, int64_t sc_interval,
               swb::BestRec *best_out, float *ms_out, int64_t *nsr_out, const BlockIo *blk = nullptr) {
    using namespace swb;
    cudaError_t e;
    // TAB mode when the column sequence has at most four distinct bytes and the
    // shifted scores fit a signed byte
    bool tab = false;
    uint8_t lut[256];
    c->last_launches = 2;  // wavefront + best-cell reduction
    const int32_t mt1 = sc->match - sc->gap_open, mm1 = sc->mismatch - sc->gap_open;
    if (mt1 >= -128 && mt1 <= 127 && mm1 >= -128 && mm1 <= 127 && !std::getenv("SWB_STAGE1_CMP")) {
        uint32_t present[256];
        if ((e = c->flags.ensure(256 * sizeof(uint32_t))) != cudaSuccess ||
            (e = stage1_presence(d_cols, n, (uint32_t *)c->flags.p, c->stream)) != cudaSuccess ||
            (e = swb::ctx_get(c, present, c->flags.p, sizeof present)) != cudaSuccess)
            return ctx_cuda_fail(c, e, "column alphabet");
        c->last_launches += 1;
        int K = 0;
        for (int i = 0; i < 256; ++i) lut[i] = present[i] ? (uint8_t)(K++) : 7;
        tab = K <= 4;
    }
    if ((e = c->hbuf.ensure(sizeof(int4) * (size_t)std::max<int64_t>(n, 1))) != cudaSuccess ||
        (e = c->best.ensure(sizeof(BestRec))) != cudaSuccess ||
        (e = c->errf.ensure(4 * sizeof(int32_t))) != cudaSuccess)
        return ctx_cuda_fail(c, e, "stage 1 buffers");

    Stage1Args a{};
    a.rows = d_rows;
    a.cols = d_cols;
    a.m = m;
    a.n = n;
    a.open = sc->gap_open;
    a.ext = sc->gap_extend;
    a.gx = std::max(sc->gap_open, sc->gap_extend);
    a.mt1 = mt1;
    a.mm1 = mm1;
    if (tab) {
        if ((e = c->lut.ensure(256)) != cudaSuccess || (e = c->rcode.ensure((size_t)m + 64)) != cudaSuccess ||
            (e = c->ctab.ensure(sizeof(uint32_t) * ((size_t)n + 64))) != cudaSuccess ||
            (e = swb::ctx_put(c, c->lut.p, lut, 256)) != cudaSuccess ||
            (e = stage1_encode(d_rows, m, d_cols, n, (const uint8_t *)c->lut.p, (uint8_t *)c->rcode.p,
                               (uint32_t *)c->ctab.p, mt1, mm1, &a.tab_hi, c->stream)) != cudaSuccess)
            return ctx_cuda_fail(c, e, "stage 1 encode");
        c->last_launches += 1;
        a.rcode = (const uint8_t *)c->rcode.p;
        a.ctab = (const uint32_t *)c->ctab.p;
    }
    a.hbuf = (int4 *)c->hbuf.p;
    a.best = (BestRec *)c->best.p;
    a.err = (int32_t *)c->errf.p;
    a.gbest = a.err + 2;
    a.wait_limit = c->wait_cycles;
    int32_t G = 0, T = 0;
    int64_t P1 = 0, P2 = 0;
    const bool refok = blk ? reference_geometry(blk->full_m, blk->full_n, &G, &T, &P1, &P2)
                           : reference_geometry(m, n, &G, &T, &P1, &P2);
    a.tie.mode = ((flags & SWB_FLAG_TIE_ROWMAJOR) || !refok) ? kTieRowMajor : kTieReference;
    a.tie.G = G;
    a.tie.T = T;
    a.tie.C = refok ? P2 / G : 1;
    if (blk) {
        a.top = blk->top;
        a.left = blk->left;
        a.corner = blk->corner;
        a.r_origin = blk->r0;
        a.c_origin = blk->c0;
        a.bottom = blk->bottom;
        a.right = blk->right;
    }

    // rows per lane: an override, else the autotuner.  Strips must tile the
    // special-row spacing when special rows are kept; sr_interval_rows < 0 asks
    // for a special row at every strip bottom with the strip height left to the
    // tuner (448 or 512 rows: the walker's block grid follows it).
    const bool strip_rows = sr_interval_rows < 0;
    const bool stores = sr_interval_rows != 0 || sc_interval > 0;
    int R = 16;
    if (blk && blk->bottom) R = 16;  // the last row must be a strip bottom: 512-row strips
    else if (const char *rv = std::getenv("SWB_STAGE1_R")) R = std::atoi(rv);  // override: 8, 14, 16 or 32
    else R = autotune_rows_per_lane(c, a, tab, stores, 16, strip_rows, sr_interval_rows > 0 ? sr_interval_rows : 0);
    if (strip_rows) {
        if (R != 14 && R != 16) R = 16;
        sr_interval_rows = 32LL * R;
    }
    if (sr_interval_rows > 0 && (R > 16 || sr_interval_rows % (32 * R) != 0)) R = 16;
    Stage1Plan plan = stage1_plan(m, n, c->sms, R, tab);
    if (c->max_blocks > 0 && plan.blocks > c->max_blocks) plan.blocks = c->max_blocks;
    const int64_t W = (int64_t)plan.blocks * plan.warps_per_block;
    if ((e = c->wbest.ensure(sizeof(BestRec) * (size_t)W)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "stage 1 buffers");
    a.nstrips = plan.nstrips;
    a.wbest = (BestRec *)c->wbest.p;
    a.srows = nullptr;
    a.sr_every = 1;
    a.nsr = 0;
    a.trace = nullptr;
    c->last_nstrips = plan.nstrips;
    if (c->opts.verbose & 2) {  // stage-1 strip trace, read back with swb_trace_copy
        if ((e = c->trace.ensure(sizeof(int64_t) * 3 * (size_t)plan.nstrips)) != cudaSuccess)
            return ctx_cuda_fail(c, e, "trace buffer");
        a.trace = (int64_t *)c->trace.p;
    }
    a.scols = nullptr;
    a.sc_every = 1 << 30;
    a.nsc = 0;
    size_t sbytes = 0;
    if (sr_interval_rows > 0) {
        const int64_t every = std::max<int64_t>(1, sr_interval_rows / plan.strip_rows);
        const int64_t nsr = (m / plan.strip_rows) / every;
        sbytes += sizeof(int2) * (size_t)nsr * (size_t)n;
        if (nsr > 0) {
            a.sr_every = every;
            a.nsr = nsr;
        }
    }
    if (sc_interval > 0) {
        const int64_t nsc = n / sc_interval;
        sbytes += sizeof(int2) * (size_t)nsc * (size_t)m;
        if (nsc > 0) {
            a.sc_every = (int32_t)sc_interval;
            a.nsc = nsc;
        }
    }
    const size_t rows_bytes = sizeof(int2) * (size_t)a.nsr * (size_t)n;
    const size_t cols_bytes = sizeof(int2) * (size_t)a.nsc * (size_t)m;
    bool rows_host = false, cols_host = false;
    if (!tb::spill_placement(c->opts.hbm_budget_bytes, c->opts.host_spill_bytes, rows_bytes, cols_bytes, &rows_host,
                             &cols_host))
        return ctx_fail(c, SWB_ENOMEM_BUDGET, "special rows and columns need %zu bytes > budget %llu + spill %llu",
                        sbytes, (unsigned long long)c->opts.hbm_budget_bytes,
                        (unsigned long long)c->opts.host_spill_bytes);
    c->last_host_bytes = (int64_t)((rows_host ? rows_bytes : 0) + (cols_host ? cols_bytes : 0));
    if (a.nsr > 0) {
        if (rows_host) {
            if ((e = c->srows_h.ensure(rows_bytes)) != cudaSuccess) return ctx_cuda_fail(c, e, "spilled special rows");
            a.srows = (int2 *)c->srows_h.dp;
        } else {
            if ((e = c->srows.ensure(rows_bytes)) != cudaSuccess) return ctx_cuda_fail(c, e, "special rows");
            a.srows = (int2 *)c->srows.p;
        }
    }
    if (a.nsc > 0) {
        if (cols_host) {
            if ((e = c->scols_h.ensure(cols_bytes)) != cudaSuccess)
                return ctx_cuda_fail(c, e, "spilled special columns");
            a.scols = (int2 *)c->scols_h.dp;
        } else {
            if ((e = c->scols.ensure(cols_bytes)) != cudaSuccess) return ctx_cuda_fail(c, e, "special columns");
            a.scols = (int2 *)c->scols.p;
        }
    }
    c->last_srows = a.srows;
    c->last_scols = a.scols;
    c->last_nsr = a.nsr;
    c->last_n = n;
    c->last_sr_interval = a.nsr > 0 ? a.sr_every * plan.strip_rows : 0;
    if (nsr_out) *nsr_out = a.nsr;

    if ((e = cudaMemsetAsync(a.hbuf, 0xFF, sizeof(int4) * (size_t)n, c->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(a.err, 0, 4 * sizeof(int32_t), c->stream)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "stage 1 reset");
    a.withhold = (flags & SWB_FLAG_TEST_WITHHOLD) ? 1 : 0;  // set after the autotuner's probes
    cudaEventRecord(c->ev0, c->stream);
    if ((e = stage1_launch(a, plan, c->stream)) != cudaSuccess) return ctx_cuda_fail(c, e, "stage 1 launch");
    cudaEventRecord(c->ev1, c->stream);
    int32_t errh[2] = {0, 0};
    if ((e = swb::ctx_get(c, best_out, a.best, sizeof(BestRec))) != cudaSuccess ||
        (e = swb::ctx_get(c, errh, a.err, sizeof errh)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "stage 1");
    if (errh[0] != 0) return ctx_fail(c, SWB_ETIMEOUT, "stage 1: a bounded wait between strips ran out");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    if (ms_out) *ms_out = ms;
    return SWB_OK;
}

int align_device(swb_ctx *c, const uint8_t *d_rows, int64_t m, const uint8_t *d_cols, int64_t n,
                 const swb_scoring *sc, uint32_t flags, swb_result *out, int swapped) {
    using namespace swb;
    const auto t0 = std::chrono::steady_clock::now();
    std::memset(out, 0, sizeof *out);
    out->rows = m;
    out->cols = n;
    out->swapped = swapped;
    int32_t G = 0, T = 0;
    int64_t P1 = 0, P2 = 0;
    reference_geometry(m, n, &G, &T, &P1, &P2);
    out->xpoint_interval = T > 0 ? 4 * T : 20;
    if (m == 0 || n == 0) {
        out->total_ms = 0;
        return SWB_OK;
    }
    const bool score_only = (flags & SWB_FLAG_SCORE_ONLY) != 0;
    tb::Plan plan;
    int64_t sr_interval = 0, sc_interval = 0;
    if (!score_only) {
        plan = tb::plan_for(c->opts, m, n);
        sr_interval = plan.kr;
        sc_interval = plan.kc;
        // direct mode, with room for special rows every 448 rows as well: the
        // strip height (448 or 512) is tuned and the walker's grid follows it
        if (!plan.level1 && !tb::plan_for(c->opts, m, n, 448).level1) sr_interval = -1;
    } else if (c->opts.special_interval > 0 && !(flags & SWB_FLAG_NO_SPECIAL)) {
        sr_interval = c->opts.special_interval;  // inspection of special rows only
    }
    BestRec best{};
    float ms = 0.f;
    int64_t nsr = 0;
    int rc = run_stage1(c, d_rows, m, d_cols, n, sc, flags, sr_interval, sc_interval, &best, &ms, &nsr);
    if (rc != SWB_OK) return rc;
    out->stage1_ms = ms;
    out->kernel_launches += c->last_launches;
    out->special_interval = (int32_t)c->last_sr_interval;
    if (!score_only && sr_interval < 0) plan = tb::plan_for(c->opts, m, n, c->last_sr_interval);
    out->special_bytes = (int64_t)sizeof(int2) * nsr * n + (sc_interval > 0 ? (int64_t)sizeof(int2) * (n / sc_interval) * m : 0);
    out->host_bytes = c->last_host_bytes;
    if (best.valid) {
        out->score = best.ho - sc->gap_open;
        out->end_row = best.row;
        out->end_col = best.col;
    } else {
        out->score = 0;
        out->end_row = 0;
        out->end_col = 0;
    }
    out->start_row = out->end_row;
    out->start_col = out->end_col;
    if (!score_only && out->score > 0) {
        const auto t1 = std::chrono::steady_clock::now();
        tb::Scratch scr;
        scr.owner = c;
        scr.ensure = [](void *owner, int which, size_t bytes) -> void * {
            swb_ctx *cx = (swb_ctx *)owner;
            return cx->tb[which].ensure(bytes) == cudaSuccess ? cx->tb[which].p : nullptr;
        };
        scr.get = [](void *owner, void *dst, const void *src, size_t bytes) -> cudaError_t {
            return swb::ctx_get((swb_ctx *)owner, dst, src, bytes);
        };
        scr.put = [](void *owner, void *dst, const void *src, size_t bytes) -> cudaError_t {
            return swb::ctx_put((swb_ctx *)owner, dst, src, bytes);
        };
        int32_t launches = 0;
        // a capped context (the serving loop's long lane) sizes its stage-2 grids
        // to the same share of the GPU as its stage 1 (4 scoring blocks per SM)
        const int tb_sms = c->max_blocks > 0 ? std::max(1, std::min(c->sms, c->max_blocks / 4)) : c->sms;
        rc = tb::traceback(c->stream, tb_sms, d_rows, m, d_cols, n, sc, plan, c->last_srows, c->last_scols, out, scr,
                           c->err, &launches);
        if (rc != SWB_OK) return ctx_fail(c, rc, "%s", c->err.c_str());
        out->kernel_launches += launches;
        out->stage2_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
    } else if (!score_only) {
        // best score 0: empty alignment, crosspoints [start = end]
        out->xpoints = (swb_xpoint *)std::malloc(sizeof(swb_xpoint) * 2);
        if (out->xpoints) {
            out->xpoints[0] = swb_xpoint{0, 0, out->end_row, out->end_col};
            out->n_xpoints = 1;
        }
    }
    out->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return SWB_OK;
}

}  // namespace

extern "C" int swb_align_pair_device(swb_ctx *c, const void *d_rows, int64_t rows, const void *d_cols, int64_t cols,
                                     const swb_scoring *sc, uint32_t flags, swb_result *out) {
    if (!c || !out || rows < 0 || cols < 0 || rows < cols || (rows > 0 && !d_rows) || (cols > 0 && !d_cols))
        return ctx_fail(c, SWB_EINVAL, "swb_align_pair_device: bad arguments");
    if (rows > (int64_t)INT32_MAX - 64 || cols > (int64_t)INT32_MAX - 64)
        return ctx_fail(c, SWB_EUNSUPPORTED, "sequence longer than 2^31 - 64");
    int rc = check_scoring(c, sc, rows, cols);
    if (rc != SWB_OK) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    return align_device(c, (const uint8_t *)d_rows, rows, (const uint8_t *)d_cols, cols, sc, flags, out, 0);
}

extern "C" int swb_score_block_device(swb_ctx *c, const void *d_rows, int64_t rows, const void *d_cols, int64_t cols,
                                      const int32_t *d_top, const int32_t *d_left, int32_t corner, int64_t row_origin,
                                      int64_t col_origin, int64_t full_rows, int64_t full_cols, const swb_scoring *sc,
                                      uint32_t flags, int32_t *d_bottom, int32_t *d_right, swb_block_best *out) {
    if (!c || !out || rows <= 0 || cols <= 0 || !d_rows || !d_cols || row_origin < 0 || col_origin < 0 ||
        full_rows < full_cols || row_origin + rows > full_rows || col_origin + cols > full_cols)
        return ctx_fail(c, SWB_EINVAL, "swb_score_block_device: bad arguments");
    if (full_rows > (int64_t)INT32_MAX - 64)
        return ctx_fail(c, SWB_EUNSUPPORTED, "sequence longer than 2^31 - 64");
    if (d_bottom && rows % 512 != 0)
        return ctx_fail(c, SWB_EINVAL, "swb_score_block_device: the bottom row needs rows to be a multiple of 512");
    int rc = check_scoring(c, sc, full_rows, full_cols);
    if (rc != SWB_OK) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    BlockIo io;
    io.top = (const int2 *)d_top;
    io.left = (const int2 *)d_left;
    io.corner = corner;
    io.r0 = row_origin;
    io.c0 = col_origin;
    io.full_m = full_rows;
    io.full_n = full_cols;
    io.bottom = (int2 *)d_bottom;
    io.right = (int2 *)d_right;
    swb::BestRec best{};
    float ms = 0.f;
    rc = run_stage1(c, (const uint8_t *)d_rows, rows, (const uint8_t *)d_cols, cols, sc,
                    flags & SWB_FLAG_TIE_ROWMAJOR, 0, 0, &best, &ms, nullptr, &io);
    if (rc != SWB_OK) return rc;
    const bool any = best.valid && best.ho - sc->gap_open > 0;
    out->score = any ? best.ho - sc->gap_open : 0;
    out->row = any ? row_origin + best.row : -1;
    out->col = any ? col_origin + best.col : -1;
    out->key = any ? best.key : ~0ULL;
    out->stage1_ms = ms;
    return SWB_OK;
}

extern "C" int swb_align_pair(swb_ctx *c, const uint8_t *a, int64_t la, const uint8_t *b, int64_t lb,
                              const swb_scoring *sc, uint32_t flags, swb_result *out) {
    if (!c || !out || la < 0 || lb < 0 || (la > 0 && !a) || (lb > 0 && !b))
        return ctx_fail(c, SWB_EINVAL, "swb_align_pair: bad arguments");
    const bool swap = la < lb;  // src/SWutils.cpp:84-88
    const uint8_t *hr = swap ? b : a;
    const uint8_t *hc = swap ? a : b;
    const int64_t m = swap ? lb : la, n = swap ? la : lb;
    if (m > (int64_t)INT32_MAX - 64)
        return ctx_fail(c, SWB_EUNSUPPORTED, "sequence longer than 2^31 - 64");
    int rc = check_scoring(c, sc, m, n);
    if (rc != SWB_OK) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    cudaError_t e;
    if ((e = c->rows.ensure((size_t)m + 64)) != cudaSuccess || (e = c->cols.ensure((size_t)n + 64)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "sequence buffers");
    if ((e = swb::ctx_put(c, c->rows.p, hr, (size_t)m)) != cudaSuccess) return ctx_cuda_fail(c, e, "copy rows");
    if ((e = swb::ctx_put(c, c->cols.p, hc, (size_t)n)) != cudaSuccess) return ctx_cuda_fail(c, e, "copy cols");
    return align_device(c, (const uint8_t *)c->rows.p, m, (const uint8_t *)c->cols.p, n, sc, flags, out, swap ? 1 : 0);
}

// Copies special row `idx` (row (idx+1)*interval - 1) of the last call as (H, F)
// pairs into host memory `out` (2*cols int32).  Inspection entry for tests.
extern "C" int swb_special_row_copy(swb_ctx *c, int64_t idx, int32_t *out, int64_t cols, int64_t *interval) {
    if (!c || !out) return ctx_fail(c, SWB_EINVAL, "swb_special_row_copy: bad arguments");
    if (interval) *interval = c->last_sr_interval;
    if (idx < 0 || idx >= c->last_nsr || cols != c->last_n)
        return ctx_fail(c, SWB_EINVAL, "special row %lld not available", (long long)idx);
    cudaSetDevice(c->device);
    cudaError_t e = swb::ctx_get(c, out, c->last_srows + idx * c->last_n, sizeof(int2) * (size_t)cols);
    if (e != cudaSuccess) return ctx_cuda_fail(c, e, "special row copy");
    return SWB_OK;
}

// Copies the stage-1 strip trace of the last call (options.verbose bit 1 set):
// per strip {start ns, end ns, SM id}.  Returns the number of strips in *count.
extern "C" int swb_trace_copy(swb_ctx *c, int64_t *out, int64_t cap, int64_t *count) {
    if (!c || !out || !count) return ctx_fail(c, SWB_EINVAL, "swb_trace_copy: bad arguments");
    *count = c->last_nstrips;
    if (!c->trace.p || cap < 3 * c->last_nstrips) return ctx_fail(c, SWB_EINVAL, "no trace or buffer too small");
    cudaSetDevice(c->device);
    cudaError_t e = swb::ctx_get(c, out, c->trace.p, sizeof(int64_t) * 3 * (size_t)c->last_nstrips);
    return e == cudaSuccess ? SWB_OK : ctx_cuda_fail(c, e, "trace copy");
}
