// autotune.cpp -- the stage-1 tile autotuner: rows per lane R (the strip height
// is 32 R rows, the cells a thread updates per column) for the pair path.
//
// The best R depends on the device, on the store mode and on how many strips a
// pair has against the warps the GPU holds (measured on the 1 Mbp pair on B200:
// R = 8 is 8% faster than R = 16 without stores; on the 10 Mbp pair with stores
// R = 16 is 25% faster than R = 8).  So the first pair of a shape bucket times
// every candidate on a slice of that pair (all its rows, up to 2^18 columns, the
// same kernel mode), keeps the fastest, and later pairs of the bucket reuse it.
// Buckets: SM count, store mode, substitution mode, ceil(log2) of rows and of
// columns.  With SWB_AUTOTUNE_CACHE=<file> the table is read at first use and
// every new entry appended, so later processes skip the probes.  The special-row
// spacing is the other tuned parameter; it is chosen from the HBM budget by the
// traceback planner (the densest grid that fits).
//
// Batches: the packed 16-bit pass takes 448- or 256-row strips.  Short pairs pad
// less with 256 rows, long ones run fewer per-strip steps with 448, so the
// choice depends on the batch's length mix.  Its bucket is the SM count and
// ceil(log2) of the cells-weighted median rows and columns of the packed pairs;
// batch_host.cpp times each candidate on a strided sample of the batch's own
// pairs (the samples' results are kept) and records the faster here, in the
// same table and file.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "ctx.h"

namespace swb {
namespace {

std::mutex g_mu;
std::map<std::string, int> g_table;
bool g_loaded = false;

int log2ceil(int64_t x) {
    int b = 0;
    while ((1LL << b) < x && b < 62) ++b;
    return b;
}

std::string key_of(int sms, bool stores, bool tab, int64_t m, int64_t n) {
    char k[96];
    snprintf(k, sizeof k, "sms%d %s %s r%d c%d", sms, stores ? "stores" : "score", tab ? "tab" : "cmp",
             log2ceil(m), log2ceil(n));
    return k;
}

void load_locked() {
    if (g_loaded) return;
    g_loaded = true;
    const char *path = std::getenv("SWB_AUTOTUNE_CACHE");
    if (!path) return;
    FILE *f = std::fopen(path, "r");
    if (!f) return;
    char line[256];
    while (std::fgets(line, sizeof line, f)) {
        char a[32], b[16], c[16], d[16], e[16];
        int R = 0;
        if (std::sscanf(line, "%31s %15s %15s %15s %15s %d", a, b, c, d, e, &R) == 6 && (R == 8 || R == 14 || R == 16 || R == 32))
            g_table[std::string(a) + " " + b + " " + c + " " + d + " " + e] = R;
    }
    std::fclose(f);
}

void store_locked(const std::string &key, int R) {
    g_table[key] = R;
    const char *path = std::getenv("SWB_AUTOTUNE_CACHE");
    if (!path) return;
    FILE *f = std::fopen(path, "a");
    if (!f) return;
    std::fprintf(f, "%s %d\n", key.c_str(), R);
    std::fclose(f);
}

}  // namespace

std::string batch_tune_key(int sms, const char *pass, int64_t m, int64_t n) {
    char k[96];
    snprintf(k, sizeof k, "sms%d %s tab r%d c%d", sms, pass, log2ceil(m), log2ceil(n));
    return k;
}

bool tune_lookup(const std::string &key, int *R) {
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    auto it = g_table.find(key);
    if (it == g_table.end()) return false;
    *R = it->second;
    return true;
}

void tune_record(const std::string &key, int R) {
    std::lock_guard<std::mutex> lk(g_mu);
    load_locked();
    store_locked(key, R);
}

int autotune_rows_per_lane(swb_ctx *c, const Stage1Args &base, bool tab, bool stores, int fallback,
                           bool strip_rows, int64_t sr_interval) {
    // pairs below this many cells are not worth a probe
    constexpr double kMinCells = 2e10;
    if ((double)base.m * (double)base.n < kMinCells) return fallback;
    const std::string key = key_of(c->sms, stores, tab, base.m, base.n) + (strip_rows ? "|strip" : "") +
                            (sr_interval > 0 ? "|sr" + std::to_string(sr_interval) : "");
    {
        std::lock_guard<std::mutex> lk(g_mu);
        load_locked();
        auto it = g_table.find(key);
        if (it != g_table.end()) return it->second;
    }
    // score only: any height; stores at every strip bottom (direct traceback): 448
    // or 512 rows; special rows at a fixed interval (level 1): heights that divide it
    std::vector<int> cands;
    if (!stores) cands = {8, 14, 16, 32};
    else if (strip_rows) cands = {14, 16};
    else
        for (int R : {8, 14, 16})
            if (sr_interval <= 0 || sr_interval % (32 * R) == 0) cands.push_back(R);
    if (cands.empty()) return fallback;
    if (stores) {
        // Launches with stores choose between 448- and 512-row strips by how well
        // the strips fill the resident warps over whole rounds: a probe on a
        // column slice of a tall pair is dominated by the wavefront's fill, which
        // favours fewer strips, while the full pair is not.  The store kernel does
        // about 4% less per cell with 512-row strips, so 448 rows must fill the
        // warps more than 4% better.  Measured with 448- vs 512-row strips: 1 Mbp
        // pair 627 vs 667 ms (fill 0.94 vs 0.82), 10 Mbp pair 46.2 vs 45.7 s
        // (fill 0.94 vs 0.92).
        auto fill = [&](int R) {
            const int per_sm = stage1_max_blocks_per_sm(R, tab);
            const double slots = (double)std::max(1, c->sms) * std::max(1, per_sm) * 4;
            const double strips = std::ceil((double)base.m / (32.0 * R));
            return strips / (std::ceil(strips / slots) * slots);
        };
        const bool has14 = std::find(cands.begin(), cands.end(), 14) != cands.end();
        const bool has16 = std::find(cands.begin(), cands.end(), 16) != cands.end();
        if (has14 && has16) return fill(14) * 0.96 > fill(16) ? 14 : 16;
        if (has16) return 16;
        if (has14) return 14;
    }
    const int64_t np = std::min<int64_t>(base.n, 1 << 18);
    int bestR = fallback;
    float bestMs = 1e30f;
    for (int R : cands) {
        Stage1Plan p = stage1_plan(base.m, np, c->sms, R, tab);
        p.stores = stores;
        if (c->max_blocks > 0 && p.blocks > c->max_blocks) p.blocks = c->max_blocks;
        const int64_t W = (int64_t)p.blocks * p.warps_per_block;
        if (c->wbest.ensure(sizeof(BestRec) * (size_t)W) != cudaSuccess) return fallback;
        Stage1Args a = base;
        a.n = np;
        a.nstrips = p.nstrips;
        a.wbest = (BestRec *)c->wbest.p;
        a.srows = nullptr;
        a.scols = nullptr;
        a.nsr = a.nsc = 0;
        a.trace = nullptr;
        if (cudaMemsetAsync(a.hbuf, 0xFF, sizeof(int4) * (size_t)np, c->stream) != cudaSuccess ||
            cudaMemsetAsync(a.err, 0, 4 * sizeof(int32_t), c->stream) != cudaSuccess ||
            cudaEventRecord(c->ev0, c->stream) != cudaSuccess || stage1_launch(a, p, c->stream) != cudaSuccess ||
            cudaEventRecord(c->ev1, c->stream) != cudaSuccess || cudaStreamSynchronize(c->stream) != cudaSuccess)
            return fallback;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        int32_t err0 = 0;
        if (ctx_get(c, &err0, a.err, sizeof err0) != cudaSuccess || err0 != 0) return fallback;
        if (ms < bestMs) {
            bestMs = ms;
            bestR = R;
        }
    }
    std::lock_guard<std::mutex> lk(g_mu);
    store_locked(key, bestR);
    return bestR;
}

}  // namespace swb
