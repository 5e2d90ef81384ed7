// ctx.h -- the library context (swb_ctx of the C ABI) and its device buffers.
// Internal to libswb200.so; shared by the pair path (api.cpp), the batched path
// (batch_host.cpp) and the serving loop (serve.cpp).
#pragma once

#include <cstdint>
#include <mutex>
#include <string>

#include "swb_internal.h"

namespace swb {

// A device allocation that grows on demand and is reused from call to call.
// Growth is stream-ordered on the owning context's stream (cudaFreeAsync /
// cudaMallocAsync): a plain cudaFree would wait for the whole device, stalling
// every other context on it (the serving loop runs two).
struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaStream_t st = nullptr;
    cudaError_t ensure(size_t bytes);
    void release();
};

// Pinned host memory mapped into the device's address space (special rows or
// columns spilled beyond the HBM budget); dp is the address kernels use.
struct MappedBuf {
    void *p = nullptr, *dp = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes);
    void release();
};

// A pinned host allocation that grows on demand.
struct HostBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes);
    void release();
};

}  // namespace swb

struct swb_ctx {
    int device = 0;
    swb_options opts{};
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    int sms = 0;
    int64_t wait_cycles = 0;  // opts.wait_limit_ms in SM clock cycles (0: the kernels' default)
    std::string err;
    swb::DevBuf rows, cols, hbuf, wbest, best, errf, srows, scols, work, flags, lut, rcode, ctab, trace;
    swb::DevBuf tb[24];  // traceback scratch (ops, crosspoints, state, level-2 stores, recompute and walker buffers)
    // batched path: sequences, encodings, descriptors, per-unit / per-pair records, stores
    swb::DevBuf b_seq, b_rcode, b_ctab, b_pairs, b_units, b_hbuf, b_gbest, b_ubest, b_pbest, b_ctl, b_srows,
        b_scols, b_walk, b_ops, b_xps, b_state, b_gdir, b_sat;
    swb::MappedBuf srows_h, scols_h;  // special rows / columns spilled to pinned host memory
    int2 *last_srows = nullptr, *last_scols = nullptr;  // where the last stage 1 kept them
    int64_t last_host_bytes = 0;
    swb::HostBuf h_stage;  // pinned staging for descriptors and results
    swb::HostBuf h_io;     // pinned staging of ctx_get / ctx_put
    // graphed batches: the call header (allocated once: the graphs hold its
    // address), packed inputs, work buffers, packed results, walker scratch, their
    // pinned staging, and the instantiated graphs by shape
    swb::DevBuf g_hdr, g_in, g_work, g_out, g_dir;
    swb::HostBuf h_gin, h_gout;
    struct GraphEntry {
        cudaGraph_t graph = nullptr;        // kept: its nodes name the exec's nodes
        cudaGraphExec_t exec = nullptr;
        cudaGraphNode_t scoring[2] = {};     // the scoring kernels (table path, compare path)
        cudaKernelNodeParams kp[2] = {};     // their launch shapes
        unsigned char set_args[256] = {};    // the BatchArgs last set on them
        bool args_valid = false;
        int traced = 0, R = 0, cap = 0, size_class = 0;
    };
    GraphEntry graphs[16];
    int graph_next = 0;                  // round-robin replacement when all entries are taken
    cudaStream_t cap_stream = nullptr;   // private stream the graphs are captured on
    cudaEvent_t ev2 = nullptr;
    int64_t last_nstrips = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::mutex mu;
    // last stage-1 special-row layout (for swb_special_row_copy)
    int64_t last_nsr = 0, last_n = 0, last_sr_interval = 0;
    int32_t last_launches = 0;  // this library's kernels launched by the last stage 1
    int32_t max_blocks = 0;     // cap on the scoring grids of this context (0 = whole GPU); set by the server

    template <class F>
    void each_buf(F f) {
        for (swb::DevBuf *b : {&rows, &cols, &hbuf, &wbest, &best, &errf, &srows, &scols, &work, &flags, &lut,
                               &rcode, &ctab, &trace, &b_seq, &b_rcode, &b_ctab, &b_pairs, &b_units, &b_hbuf,
                               &b_gbest, &b_ubest, &b_pbest, &b_ctl, &b_srows, &b_scols, &b_walk, &b_ops, &b_xps,
                               &b_state, &b_gdir, &b_sat, &g_hdr, &g_in, &g_work, &g_out, &g_dir})
            f(*b);
        for (swb::DevBuf &b : tb) f(b);
    }
};

namespace swb {

// Timestamped trace lines on stderr when SWB_SERVE_TRACE is set (milliseconds
// since the first call): serving iterations, long requests, buffer growth.
double trace_now_ms();
bool trace_on();

// Records a one-line error on the context (and the calling thread) and returns code.
int ctx_fail(swb_ctx *ctx, int code, const char *fmt, ...);
int ctx_cuda_fail(swb_ctx *ctx, cudaError_t e, const char *what);

// Host <-> device copies of the context, always through its pinned staging
// buffer on its stream.  A copy to or from pageable host memory is synchronous in
// the driver and can hold up other threads' CUDA calls until the copy's stream
// drains (for a long scoring launch, seconds); with pinned staging a thread
// waits in cudaStreamSynchronize on its own stream only.
// ctx_get: waits for the stream, then copies bytes from device src into dst.
// ctx_put: waits for the stream (the staging buffer may feed an earlier put),
//          copies src into staging and queues the transfer to device dst.
cudaError_t ctx_get(swb_ctx *c, void *dst, const void *dev_src, size_t bytes);
cudaError_t ctx_put(swb_ctx *c, void *dev_dst, const void *src, size_t bytes);

// Rows per lane for the pair path's stage 1 (autotune.cpp): a cached choice for
// the pair's shape bucket, else timed probes of every candidate on a slice of the
// pair described by `base` (rows, columns, encodings, scoring and the hand-off,
// best and error buffers must be set).  Small pairs get `fallback`.
// strip_rows: special rows at every strip bottom, height 448 or 512 rows.
// sr_interval: special rows every that many rows (level 1), 0 for none.
int autotune_rows_per_lane(swb_ctx *c, const Stage1Args &base, bool tab, bool stores, int fallback,
                           bool strip_rows = false, int64_t sr_interval = 0);

// The autotuner's table for batched passes: the bucket key of a pass over pairs
// whose cells-weighted median is m rows by n columns, a cached choice for it
// (also read from SWB_AUTOTUNE_CACHE) and the recording of a new one.
std::string batch_tune_key(int sms, const char *pass, int64_t m, int64_t n);
bool tune_lookup(const std::string &key, int *R);
void tune_record(const std::string &key, int R);

}  // namespace swb
