// serve.cpp -- the serving loop (swb_server_*): continuous batching of
// alignment requests under an HBM admission budget.  No counterpart in the
// reference (one pair per process, src/main.cu:102-249).
//
// Two lanes, each a host thread with its own context (stream and buffers):
//   * short lane: iterations.  An iteration takes every queued short request
//     that fits the budget (up to max_batch), packs their sequences into one
//     host buffer and runs one batched scoring launch that keeps every pair's
//     special rows and columns, then one batched traceback launch.  Requests
//     that arrive meanwhile wait for the next iteration.
//   * long lane: one long request at a time through the pair path, with its
//     scoring grid capped so that reserve_sms SMs stay free for the short
//     iterations (which cap their own grid to those SMs while a long request is
//     queued or running); the two lanes' kernels run side by side.
// Admission: a request is admitted when its footprint (sequences, encodings,
// row hand-off buffer, special rows/columns and traceback buffers) fits the
// budget next to the requests already running; a request larger than the whole
// budget is refused at submission.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.h"
#include "ctx.h"
#include "traceback.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point t0, Clock::time_point t1) {
    return std::chrono::duration<double, std::milli>(t1 - t0).count();
}

struct Request {
    uint64_t id = 0;
    std::vector<uint8_t> a, b;
    int64_t m = 0, n = 0;   // rows (longer) and cols
    bool is_long = false;
    uint64_t foot = 0;
    int state = 0;          // 0 queued, 1 running, 2 finished
    int rc = SWB_OK;
    std::string err;
    swb_result res{};
    Clock::time_point t_submit, t_start, t_end;
    int32_t batch_size = 0;
};

// Device bytes a short request holds while it runs (batched path with stores).
uint64_t short_footprint(int64_t m, int64_t n) {
    const uint64_t seq = 6ULL * (uint64_t)(m + n);                       // bytes, codes, table words
    const uint64_t hbuf = 16ULL * (uint64_t)n;
    const uint64_t stores = 8ULL * ((uint64_t)(m / 512) * n + (uint64_t)(n / 256) * m);
    const uint64_t tb = (uint64_t)(m + n + 8) + 32ULL * (uint64_t)(m / 4 + 8);
    return seq + hbuf + stores + tb + 4096;
}

// Device bytes a long request holds: the pair path's buffers with its special
// rows / columns sized to `store_budget`.
uint64_t long_footprint(int64_t m, int64_t n, uint64_t store_budget, int sms) {
    swb_options o;
    swb_options_default(&o);
    o.hbm_budget_bytes = store_budget;
    const swb::tb::Plan p = swb::tb::plan_for(o, m, n);
    const uint64_t stores = 8ULL * ((uint64_t)(m / p.kr) * n + (uint64_t)(n / p.kc) * m);
    const uint64_t level2 = p.level1 ? (uint64_t)swb::tb::level1_corridor_cells(p, sms) *
                                           (uint64_t)swb::tb::level1_cell_store_bytes(p)
                                     : 0;
    const uint64_t walker = (uint64_t)4 * 148 * 4 * (256 + 31) * 32 * 4;  // precomputed direction blocks
    return 6ULL * (uint64_t)(m + n) + 16ULL * (uint64_t)n + stores + level2 + walker + (uint64_t)(m + n + 8) +
           (64ULL << 20);
}

}  // namespace

struct swb_server {
    swb_ctx *cs = nullptr, *cl = nullptr;
    swb_scoring sc{};
    swb_server_options o{};
    uint64_t long_store_budget = 0;
    int sms = 0, per_sm = 4;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> qs, ql;
    std::unordered_map<uint64_t, Request *> reqs;
    uint64_t next_id = 1;
    uint64_t reserved = 0;
    bool stop = false;
    bool long_active = false;
    std::thread ts, tl;
    swb_server_stats stats{};
    std::string err;

    void finish(Request *r, int rc, const std::string &msg) {
        // mu held
        r->rc = rc;
        r->err = msg;
        r->state = 2;
        r->t_end = Clock::now();
        reserved -= r->foot;
        stats.completed += 1;
        if (rc != SWB_OK) stats.failed += 1;
        else stats.cells_completed += r->m * r->n;
    }

    void short_lane() {
        std::vector<Request *> it;
        std::vector<uint8_t> buf;
        std::vector<swb_pair_ref> refs;
        for (;;) {
            it.clear();
            bool cap_grid = false;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return stop || !qs.empty(); });
                if (stop && qs.empty()) return;
                while (!qs.empty() && (int)it.size() < o.max_batch) {
                    Request *r = qs.front();
                    if (reserved + r->foot > o.hbm_budget_bytes && !it.empty()) break;
                    if (reserved + r->foot > o.hbm_budget_bytes) {
                        // wait for memory held by the long lane
                        cv_work.wait(lk, [&] { return stop || reserved + r->foot <= o.hbm_budget_bytes; });
                        if (stop) return;
                    }
                    qs.pop_front();
                    reserved += r->foot;
                    stats.peak_reserved_bytes = std::max<uint64_t>(stats.peak_reserved_bytes, reserved);
                    r->state = 1;
                    r->t_start = Clock::now();
                    it.push_back(r);
                }
                cap_grid = long_active || !ql.empty();
                stats.iterations += 1;
                stats.max_batch_seen = std::max<int64_t>(stats.max_batch_seen, (int64_t)it.size());
            }
            if (it.empty()) continue;
            // one host buffer for the iteration
            size_t bytes = 0;
            for (Request *r : it) bytes += r->a.size() + r->b.size();
            buf.resize(std::max<size_t>(bytes, 1));
            refs.resize(it.size());
            size_t off = 0;
            for (size_t k = 0; k < it.size(); ++k) {
                Request *r = it[k];
                std::memcpy(buf.data() + off, r->a.data(), r->a.size());
                refs[k].a_off = (int64_t)off;
                refs[k].a_len = (int64_t)r->a.size();
                off += r->a.size();
                std::memcpy(buf.data() + off, r->b.data(), r->b.size());
                refs[k].b_off = (int64_t)off;
                refs[k].b_len = (int64_t)r->b.size();
                off += r->b.size();
            }
            cs->max_blocks = cap_grid ? per_sm * o.reserve_sms : 0;
            const double tr0 = swb::trace_on() ? swb::trace_now_ms() : 0.0;
            swb_batch_result br{};
            const int rc = swb::batch_align_all_traced(cs, buf.data(), (int64_t)bytes, refs.data(), (int64_t)it.size(),
                                                       &sc, o.flags, &br);
            const std::string msg = rc == SWB_OK ? std::string() : std::string(swb_last_error(cs));
            std::vector<swb_result> res(it.size());
            int out_rc = rc;
            if (rc == SWB_OK) {
                for (size_t k = 0; k < it.size() && out_rc == SWB_OK; ++k) {
                    const swb_batch_item &b = br.items[k];
                    swb_result &x = res[k];
                    std::memset(&x, 0, sizeof x);
                    x.score = b.score;
                    x.end_row = b.end_row;
                    x.end_col = b.end_col;
                    x.start_row = b.start_row;
                    x.start_col = b.start_col;
                    x.swapped = b.swapped;
                    x.rows = it[k]->m;
                    x.cols = it[k]->n;
                    x.stage1_ms = br.stage1_ms;
                    x.stage2_ms = br.stage2_ms;
                    x.xpoint_interval = b.xpoint_interval;
                    x.special_interval = 512;
                    x.kernel_launches = br.kernel_launches;
                    if (b.n_ops > 0) {
                        x.ops = (char *)std::malloc((size_t)b.n_ops + 1);
                        if (!x.ops) out_rc = SWB_ENOMEM;
                        else {
                            std::memcpy(x.ops, br.ops + b.ops_off, (size_t)b.n_ops);
                            x.ops[b.n_ops] = 0;
                            x.n_ops = b.n_ops;
                        }
                    }
                    if (b.n_xpoints > 0 && out_rc == SWB_OK) {
                        x.xpoints = (swb_xpoint *)std::malloc(sizeof(swb_xpoint) * (size_t)b.n_xpoints);
                        if (!x.xpoints) out_rc = SWB_ENOMEM;
                        else {
                            std::memcpy(x.xpoints, br.xpoints + b.xp_off, sizeof(swb_xpoint) * (size_t)b.n_xpoints);
                            x.n_xpoints = b.n_xpoints;
                        }
                    }
                }
            }
            swb_batch_result_free(&br);
            if (swb::trace_on())
                std::fprintf(stderr, "swb trace %.1f short %zu pairs %.1f ms (cap %d)\n", tr0, it.size(),
                             swb::trace_now_ms() - tr0, cs->max_blocks);
            {
                std::lock_guard<std::mutex> lk(mu);
                for (size_t k = 0; k < it.size(); ++k) {
                    Request *r = it[k];
                    r->batch_size = (int32_t)it.size();
                    if (out_rc == SWB_OK) r->res = res[k];
                    else swb_result_free(&res[k]);
                    finish(r, out_rc, out_rc == SWB_OK ? std::string() : (msg.empty() ? "out of host memory" : msg));
                }
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
    }

    void long_lane() {
        for (;;) {
            Request *r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] {
                    return stop || (!ql.empty() && reserved + ql.front()->foot <= o.hbm_budget_bytes);
                });
                if (stop) return;
                r = ql.front();
                ql.pop_front();
                reserved += r->foot;
                stats.peak_reserved_bytes = std::max<uint64_t>(stats.peak_reserved_bytes, reserved);
                r->state = 1;
                r->t_start = Clock::now();
                long_active = true;
            }
            cl->max_blocks = std::max(1, per_sm * (sms - o.reserve_sms));
            swb_result res{};
            const int rc = swb_align_pair(cl, r->a.data(), (int64_t)r->a.size(), r->b.data(), (int64_t)r->b.size(), &sc,
                                          o.flags, &res);
            const std::string msg = rc == SWB_OK ? std::string() : std::string(swb_last_error(cl));
            if (swb::trace_on())
                std::fprintf(stderr, "swb trace %.1f long %lld x %lld stage1 %.1f stage2 %.1f total %.1f ms\n",
                             swb::trace_now_ms() - res.total_ms, (long long)r->m, (long long)r->n, res.stage1_ms,
                             res.stage2_ms, res.total_ms);
            {
                std::lock_guard<std::mutex> lk(mu);
                long_active = false;
                r->batch_size = 1;
                if (rc == SWB_OK) r->res = res;
                else swb_result_free(&res);
                stats.long_completed += rc == SWB_OK ? 1 : 0;
                finish(r, rc, msg);
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
    }
};

extern "C" {

void swb_server_options_default(swb_server_options *o) {
    std::memset(o, 0, sizeof *o);
}

int swb_server_create(const swb_server_options *opts, const swb_scoring *sc, swb_server **out) {
    if (!out || !sc) return swb::ctx_fail(nullptr, SWB_EINVAL, "swb_server_create: bad arguments");
    *out = nullptr;
    if (sc->match < 1 || sc->mismatch > -1 || sc->gap_open > -1 || sc->gap_extend > -1)
        return swb::ctx_fail(nullptr, SWB_EINVAL, "One or more scoring values were not usable!");
    swb_server *s = new (std::nothrow) swb_server();
    if (!s) return swb::ctx_fail(nullptr, SWB_ENOMEM, "out of host memory");
    if (opts) s->o = *opts;
    if (s->o.hbm_budget_bytes == 0) s->o.hbm_budget_bytes = 64ULL << 30;
    if (s->o.long_cells <= 0) s->o.long_cells = 1LL << 32;
    if (s->o.max_batch <= 0) s->o.max_batch = 8192;
    if (s->o.reserve_sms <= 0) s->o.reserve_sms = 4;  // 16 left short p99 the same and the long lane 4.5% slower
    s->sc = *sc;
    s->long_store_budget = s->o.hbm_budget_bytes / 2;
    swb_options co;
    swb_options_default(&co);
    co.device = s->o.device;
    co.hbm_budget_bytes = s->o.hbm_budget_bytes;
    int rc = swb_ctx_create(&co, &s->cs);
    if (rc == SWB_OK) {
        co.hbm_budget_bytes = s->long_store_budget;
        rc = swb_ctx_create(&co, &s->cl);
    }
    if (rc != SWB_OK) {
        if (s->cs) swb_ctx_destroy(s->cs);
        delete s;
        return rc;
    }
    // Device memory mapped up front.  Buffers grow stream-ordered (cudaMallocAsync),
    // but a growth the device's pool cannot serve from memory it already holds
    // maps new memory, which took 0.2 - 1.1 s for the long lane's 19 - 33 GB
    // special-row buffers and held up the short lane's launches meanwhile (the
    // serving loop's short-request tail).  So the pool keeps what is freed
    // (release threshold: never) and is grown once, here, to the admission budget.
    {
        cudaMemPool_t pool;
        uint64_t keep = ~0ULL;
        void *warm = nullptr;
        cudaSetDevice(s->o.device);
        if (cudaDeviceGetDefaultMemPool(&pool, s->o.device) == cudaSuccess &&
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) == cudaSuccess &&
            cudaMallocAsync(&warm, (size_t)s->o.hbm_budget_bytes, s->cl->stream) == cudaSuccess) {
            cudaFreeAsync(warm, s->cl->stream);
            cudaStreamSynchronize(s->cl->stream);
        } else {
            cudaGetLastError();  // not fatal: buffers then grow on demand as before
        }
    }
    // pinned staging sized up front: growing it later (cudaFreeHost) would stall the device
    if (s->cs->h_io.ensure(64ULL << 20) != cudaSuccess || s->cl->h_io.ensure(64ULL << 20) != cudaSuccess ||
        s->cs->h_stage.ensure(16ULL << 20) != cudaSuccess) {
        swb_ctx_destroy(s->cs);
        swb_ctx_destroy(s->cl);
        delete s;
        return swb::ctx_fail(nullptr, SWB_ENOMEM, "server: pinned staging buffers");
    }
    s->sms = s->cs->sms;
    if (s->o.reserve_sms >= s->sms) s->o.reserve_sms = std::max(1, s->sms / 8);
    s->per_sm = std::max(1, swb::batch_max_blocks_per_sm(true, swb::kBatchStores));
    s->ts = std::thread([s] { s->short_lane(); });
    s->tl = std::thread([s] { s->long_lane(); });
    *out = s;
    return SWB_OK;
}

int swb_server_submit(swb_server *s, const uint8_t *a, int64_t la, const uint8_t *b, int64_t lb, uint64_t *id) {
    if (!s || !id || la < 0 || lb < 0 || (la > 0 && !a) || (lb > 0 && !b))
        return swb::ctx_fail(nullptr, SWB_EINVAL, "swb_server_submit: bad arguments");
    if (std::max(la, lb) > (int64_t)INT32_MAX - 64)
        return swb::ctx_fail(nullptr, SWB_EUNSUPPORTED, "sequence longer than 2^31 - 64");
    Request *r = new (std::nothrow) Request();
    if (!r) return swb::ctx_fail(nullptr, SWB_ENOMEM, "out of host memory");
    try {
        r->a.assign(a, a + la);
        r->b.assign(b, b + lb);
    } catch (...) {
        delete r;
        return swb::ctx_fail(nullptr, SWB_ENOMEM, "out of host memory");
    }
    r->m = std::max(la, lb);
    r->n = std::min(la, lb);
    r->is_long = r->m * r->n > s->o.long_cells;
    r->foot = r->is_long ? long_footprint(r->m, r->n, s->long_store_budget, s->sms) : short_footprint(r->m, r->n);
    r->t_submit = Clock::now();
    if (r->foot > s->o.hbm_budget_bytes) {
        const uint64_t f = r->foot;
        delete r;
        return swb::ctx_fail(nullptr, SWB_ENOMEM_BUDGET, "request needs %llu bytes > server budget %llu",
                             (unsigned long long)f, (unsigned long long)s->o.hbm_budget_bytes);
    }
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) {
            delete r;
            return swb::ctx_fail(nullptr, SWB_EBUSY, "server is stopping");
        }
        r->id = s->next_id++;
        s->reqs[r->id] = r;
        (r->is_long ? s->ql : s->qs).push_back(r);
        s->stats.submitted += 1;
        *id = r->id;
    }
    s->cv_work.notify_all();
    return SWB_OK;
}

int swb_server_wait(swb_server *s, uint64_t id, int64_t timeout_ms, swb_result *out, swb_request_info *info) {
    if (!s || !out) return swb::ctx_fail(nullptr, SWB_EINVAL, "swb_server_wait: bad arguments");
    std::memset(out, 0, sizeof *out);
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return swb::ctx_fail(nullptr, SWB_ENOTFOUND, "unknown request %llu", (unsigned long long)id);
    Request *r = it->second;
    auto done = [&] { return r->state == 2; };
    if (timeout_ms < 0) s->cv_done.wait(lk, done);
    else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) return SWB_ETIMEOUT;
    if (info) {
        info->queued_ms = ms_since(r->t_submit, r->t_start);
        info->run_ms = ms_since(r->t_start, r->t_end);
        info->total_ms = ms_since(r->t_submit, r->t_end);
        info->lane = r->is_long ? 1 : 0;
        info->batch_size = r->batch_size;
    }
    const int rc = r->rc;
    if (rc == SWB_OK) {
        *out = r->res;
        out->total_ms = ms_since(r->t_start, r->t_end);
    } else {
        s->err = r->err;
    }
    s->reqs.erase(it);
    delete r;
    return rc;
}

int swb_server_stats_get(swb_server *s, swb_server_stats *st) {
    if (!s || !st) return SWB_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    *st = s->stats;
    return SWB_OK;
}

const char *swb_server_last_error(swb_server *s) { return s ? s->err.c_str() : ""; }

void swb_server_destroy(swb_server *s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        // queued requests are dropped; running ones finish
        for (Request *r : s->qs) s->reqs.erase(r->id), delete r;
        for (Request *r : s->ql) s->reqs.erase(r->id), delete r;
        s->qs.clear();
        s->ql.clear();
    }
    s->cv_work.notify_all();
    if (s->ts.joinable()) s->ts.join();
    if (s->tl.joinable()) s->tl.join();
    for (auto &kv : s->reqs) {
        swb_result_free(&kv.second->res);
        delete kv.second;
    }
    swb_ctx_destroy(s->cs);
    swb_ctx_destroy(s->cl);
    delete s;
}

}  // extern "C"
