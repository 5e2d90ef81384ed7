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
struct DevBuf {
    void *p = nullptr;
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
    std::string err;
    swb::DevBuf rows, cols, hbuf, wbest, best, errf, srows, scols, work, flags, lut, rcode, ctab, trace;
    swb::DevBuf tb[16];  // traceback scratch (ops, crosspoints, state, level-2 stores, recompute and walker buffers)
    // batched path: sequences, encodings, descriptors, per-unit / per-pair records, stores
    swb::DevBuf b_seq, b_rcode, b_ctab, b_pairs, b_units, b_hbuf, b_gbest, b_ubest, b_pbest, b_ctl, b_srows,
        b_scols, b_walk, b_ops, b_xps, b_state;
    swb::HostBuf h_stage;  // pinned staging for descriptors and results
    int64_t last_nstrips = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::mutex mu;
    // last stage-1 special-row layout (for swb_special_row_copy)
    int64_t last_nsr = 0, last_n = 0, last_sr_interval = 0;
    int32_t last_launches = 0;  // this library's kernels launched by the last stage 1
    int32_t max_blocks = 0;     // cap on the scoring grids of this context (0 = whole GPU); set by the server
};

namespace swb {

// Records a one-line error on the context (and the calling thread) and returns code.
int ctx_fail(swb_ctx *ctx, int code, const char *fmt, ...);
int ctx_cuda_fail(swb_ctx *ctx, cudaError_t e, const char *what);

}  // namespace swb
