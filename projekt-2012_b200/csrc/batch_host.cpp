// batch_host.cpp -- the batched entry points (swb_batch_align*): orientation,
// work-unit layout, the scoring launch, and for the best-scoring pairs a store
// pass plus the batched walker.  No counterpart in the reference (one pair per
// process, src/main.cu:102-249).
#include <algorithm>
#include <cstddef>
#include <chrono>
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <thread>
#include <utility>
#include <vector>

#include "batch.h"
#include "ctx.h"
#include "traceback.h"

namespace swb {
namespace {

struct PairInfo {
    int64_t row_off, col_off;
    int64_t m, n;
    int32_t swapped;
};

// Stable sort of idx by key(idx) descending, the order std::stable_sort gives
// with `key(x) > key(y)`: a least-significant-digit radix sort on 11-bit digits
// with as many passes as the largest key needs (100,000 pairs: about 1 ms; the
// comparison sort took 10 - 15 ms of host time per batch).
template <class Key>
void sort_desc(std::vector<int64_t> &idx, Key key) {
    const size_t n = idx.size();
    if (n < 2) return;
    std::vector<uint64_t> k(n), k2(n);
    std::vector<int64_t> i2(n);
    uint64_t mx = 0;
    for (size_t q = 0; q < n; ++q) {
        k[q] = key(idx[q]);
        mx = std::max(mx, k[q]);
    }
    for (size_t q = 0; q < n; ++q) k[q] = mx - k[q];  // ascending in mx - key
    std::vector<size_t> cnt(2049);
    for (int shift = 0; shift < 64 && (mx >> shift) != 0; shift += 11) {
        std::fill(cnt.begin(), cnt.end(), 0);
        for (size_t q = 0; q < n; ++q) ++cnt[((k[q] >> shift) & 2047) + 1];
        for (int b = 0; b < 2048; ++b) cnt[(size_t)b + 1] += cnt[(size_t)b];
        for (size_t q = 0; q < n; ++q) {
            const size_t d = cnt[(k[q] >> shift) & 2047]++;
            k2[d] = k[q];
            i2[d] = idx[q];
        }
        k.swap(k2);
        idx.swap(i2);
    }
}

// Lays out the units of `order` (indices into info, already sorted) as one
// launch: unit0 / ufirst / ucount / hbuf offsets; returns the unit count.
// extent (optional, one per entry of order): compute only the top-left
// rows x cols of the pair; the tie rule keeps the whole pair's geometry.
int64_t layout_units(const std::vector<PairInfo> &info, const std::vector<int64_t> &order, uint32_t flags,
                     int strip_rows, std::vector<BatchPair> &bp, std::vector<int32_t> &unit_pair,
                     int64_t *hbuf_entries, const std::vector<std::pair<int64_t, int64_t>> *extent = nullptr) {
    bp.resize(order.size());
    unit_pair.clear();
    int64_t units = 0, hb = 0;
    for (size_t k = 0; k < order.size(); ++k) {
        const PairInfo &p = info[(size_t)order[k]];
        BatchPair &d = bp[k];
        std::memset(&d, 0, sizeof d);
        d.row_off = p.row_off;
        d.col_off = p.col_off;
        const int64_t em = extent ? (*extent)[k].first : p.m, en = extent ? (*extent)[k].second : p.n;
        d.m = (int32_t)em;
        d.n = (int32_t)en;
        d.nstrips = (int32_t)((em + strip_rows - 1) / strip_rows);
        d.unit0 = (int32_t)units;
        d.ufirst = (int32_t)units;
        d.ucount = d.nstrips;
        d.slot = (int32_t)k;
        d.sr_every = 1;
        d.sc_every = 1 << 30;
        if (d.nstrips > 1) {
            d.hbuf_off = hb;
            hb += en;
        }
        int32_t G = 0, T = 0;
        int64_t P1 = 0, P2 = 0;
        const bool refok = reference_geometry(p.m, p.n, &G, &T, &P1, &P2);
        d.tie.mode = ((flags & SWB_FLAG_TIE_ROWMAJOR) || !refok) ? kTieRowMajor : kTieReference;
        d.tie.G = G;
        d.tie.T = T;
        d.tie.C = refok ? P2 / G : 1;
        for (int32_t s = 0; s < d.nstrips; ++s) unit_pair.push_back((int32_t)k);
        units += d.nstrips;
    }
    *hbuf_entries = hb;
    return units;
}

// Claim order of a launch's strips: pairs whose own chain (n columns plus the
// hand-off lag of every strip) is at least half of one warp's share of the
// launch pair by pair, first; the others strip-major (strip 0 of each, then
// strip 1, ...), so that a strip is seldom claimed before the strip above it is
// far enough ahead.  Every strip comes after the one it waits for.  Appends
// (pair, strip) to up / us; nstrips[k], n[k]: pair k's strips and columns.
void claim_order(const std::vector<int32_t> &nstrips, const std::vector<int32_t> &n, double share_steps,
                 std::vector<int32_t> &up, std::vector<int32_t> &us) {
    constexpr double kLagSteps = 84.0;
    std::vector<int32_t> flow;
    for (size_t k = 0; k < nstrips.size(); ++k) {
        if (2.0 * ((double)n[k] + (nstrips[k] - 1) * kLagSteps) >= share_steps) {
            for (int32_t s = 0; s < nstrips[k]; ++s) {
                up.push_back((int32_t)k);
                us.push_back(s);
            }
        } else {
            flow.push_back((int32_t)k);
        }
    }
    std::stable_sort(flow.begin(), flow.end(), [&](int32_t x, int32_t y) { return nstrips[x] > nstrips[y]; });
    for (int32_t s = 0; !flow.empty() && s < nstrips[(size_t)flow[0]]; ++s)
        for (size_t i = 0; i < flow.size() && nstrips[(size_t)flow[i]] > s; ++i) {
            up.push_back(flow[i]);
            us.push_back(s);
        }
}

// Runs one scoring launch (optionally the store pass) over bp; pbest receives
// one record per entry of bp (slot k).  strip_major: claim the strips in
// claim_order instead of pair by pair.
int run_launch(swb_ctx *c, const uint8_t *d_seq, bool tab, const BatchArgs &base, std::vector<BatchPair> &bp,
               std::vector<int32_t> &unit_pair, int64_t hbuf_entries, bool stores, int R, std::vector<BestRec> &pbest,
               float *ms, bool strip_major = false) {
    cudaError_t e;
    const int64_t np = (int64_t)bp.size(), nu = (int64_t)unit_pair.size();
    std::vector<int32_t> us;
    if (strip_major && np > 0) {
        std::vector<int32_t> ns((size_t)np), nc((size_t)np), up;
        double rect = 0.0;
        for (int64_t k = 0; k < np; ++k) {
            ns[(size_t)k] = bp[(size_t)k].nstrips;
            nc[(size_t)k] = bp[(size_t)k].n;
            rect += (double)bp[(size_t)k].m * (double)bp[(size_t)k].n;
        }
        const int warps = std::max(1, batch_resident_warps(tab, stores ? kBatchStores : kBatchScore, c->sms,
                                                          c->max_blocks));
        up.reserve((size_t)nu);
        us.reserve((size_t)nu);
        claim_order(ns, nc, rect / warps / (32.0 * R), up, us);
        unit_pair.swap(up);
    }
    const size_t bp_bytes = sizeof(BatchPair) * (size_t)np, up_bytes = sizeof(int32_t) * (size_t)nu * (us.empty() ? 1 : 2);
    if ((e = c->b_pairs.ensure(bp_bytes)) != cudaSuccess || (e = c->b_units.ensure(up_bytes)) != cudaSuccess ||
        (e = c->b_hbuf.ensure(sizeof(int4) * (size_t)std::max<int64_t>(1, hbuf_entries))) != cudaSuccess ||
        (e = c->b_gbest.ensure(sizeof(int32_t) * (size_t)np)) != cudaSuccess ||
        (e = c->b_ubest.ensure(sizeof(BestRec) * (size_t)std::max<int64_t>(1, nu))) != cudaSuccess ||
        (e = c->b_pbest.ensure(sizeof(BestRec) * (size_t)np)) != cudaSuccess ||
        (e = c->b_ctl.ensure(4 * sizeof(int32_t))) != cudaSuccess ||
        (e = c->h_stage.ensure(std::max(bp_bytes + up_bytes, sizeof(BestRec) * (size_t)np + 64) + 64)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "batch buffers");
    // descriptors through pinned staging (one buffer, two copies)
    uint8_t *hs = (uint8_t *)c->h_stage.p;
    std::memcpy(hs, bp.data(), bp_bytes);
    std::memcpy(hs + bp_bytes, unit_pair.data(), sizeof(int32_t) * (size_t)nu);
    if (!us.empty()) std::memcpy(hs + bp_bytes + sizeof(int32_t) * (size_t)nu, us.data(), sizeof(int32_t) * (size_t)nu);
    BatchArgs a = base;
    a.seq = d_seq;
    a.cseq = d_seq;
    a.pairs = (const BatchPair *)c->b_pairs.p;
    a.unit_pair = (const int32_t *)c->b_units.p;
    a.unit_strip = us.empty() ? nullptr : (const int32_t *)c->b_units.p + nu;
    a.nunits = nu;
    a.hbuf = (int4 *)c->b_hbuf.p;
    a.gbest = (int32_t *)c->b_gbest.p;
    a.ubest = (BestRec *)c->b_ubest.p;
    a.ctl = (int32_t *)c->b_ctl.p;
    if ((e = cudaMemcpyAsync(c->b_pairs.p, hs, bp_bytes, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(c->b_units.p, hs + bp_bytes, up_bytes, cudaMemcpyHostToDevice, c->stream)) !=
            cudaSuccess ||
        (hbuf_entries > 0 &&
         (e = cudaMemsetAsync(a.hbuf, 0xFF, sizeof(int4) * (size_t)hbuf_entries, c->stream)) != cudaSuccess) ||
        (e = cudaMemsetAsync(a.gbest, 0, sizeof(int32_t) * (size_t)np, c->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->b_pbest.p, 0, sizeof(BestRec) * (size_t)np, c->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(a.ctl, 0, 4 * sizeof(int32_t), c->stream)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "batch set-up");
    cudaEventRecord(c->ev0, c->stream);
    if ((e = batch_launch(a, tab, stores ? kBatchStores : kBatchScore, R, c->sms, c->max_blocks, np,
                          (BestRec *)c->b_pbest.p, c->stream)) !=
        cudaSuccess)
        return ctx_cuda_fail(c, e, "batch launch");
    cudaEventRecord(c->ev1, c->stream);
    int32_t ctl[4] = {0, 0, 0, 0};
    pbest.resize((size_t)np);
    int32_t *hctl = (int32_t *)(hs + sizeof(BestRec) * (size_t)np);  // pinned, after the records
    if ((e = cudaMemcpyAsync(hs, c->b_pbest.p, sizeof(BestRec) * (size_t)np, cudaMemcpyDeviceToHost, c->stream)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(hctl, a.ctl, sizeof ctl, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c->stream)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "batch");
    std::memcpy(ctl, hctl, sizeof ctl);
    if (ctl[1] != 0) return ctx_fail(c, SWB_ETIMEOUT, "batch: a bounded wait between strips ran out");
    std::memcpy(pbest.data(), hs, sizeof(BestRec) * (size_t)np);
    float t = 0.f;
    cudaEventElapsedTime(&t, c->ev0, c->ev1);
    if (ms) *ms += t;
    return SWB_OK;
}

// Store offsets of the traced pairs `bp` (special rows every 512 rows, special
// columns every 256 columns) and the output capacities; returns the total
// store entries in *srn / *scn.
void layout_stores(std::vector<BatchPair> &bp, const swb_batch_item *items, const std::vector<int64_t> &idx,
                   int64_t *srn, int64_t *scn, int64_t *ops_total, int64_t *xp_total) {
    const int kBC = tb::block_cols();
    *srn = *scn = *ops_total = *xp_total = 0;
    for (size_t k = 0; k < bp.size(); ++k) {
        BatchPair &d = bp[k];
        d.sr_every = 1;
        d.sc_every = kBC;
        d.sr_off = *srn;
        d.sc_off = *scn;
        *srn += (int64_t)(d.m / kBatchStripRows) * d.n;
        *scn += (int64_t)(d.n / kBC) * d.m;
        *ops_total += (int64_t)d.m + d.n + 8;
        *xp_total += d.m / items[idx[k]].xpoint_interval + 8;
    }
}


// Host copy into pinned staging, split over a few threads for large buffers
// (one core copies ~10 GB/s; the batch's sequences are tens of MB).
void copy_parallel(uint8_t *dst, const uint8_t *src, size_t bytes) {
    constexpr size_t kChunk = 8u << 20;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t parts = std::min<size_t>(std::min<size_t>(8, hw), (bytes + kChunk - 1) / kChunk);
    if (parts <= 1) {
        if (bytes) std::memcpy(dst, src, bytes);
        return;
    }
    const size_t per = (bytes + parts - 1) / parts;
    std::vector<std::thread> th;
    for (size_t k = 1; k < parts; ++k) {
        const size_t lo = k * per, n = lo < bytes ? std::min(per, bytes - lo) : 0;
        if (n) th.emplace_back([=] { std::memcpy(dst + lo, src + lo, n); });
    }
    std::memcpy(dst, src, std::min(per, bytes));
    for (auto &t : th) t.join();
}

bool graphs_enabled() {
    const char *v = std::getenv("SWB_BATCH_GRAPH");
    return !(v && v[0] == '0');
}

// The packed 16-bit scoring pass (batch16.cu) serves score-only passes of
// batches with at least this many pairs in the table (<= 4 letter) mode; the
// smaller batches of the serving loop keep the replayed graph.
constexpr int64_t kPackMinPairs = 2048;

bool packing_enabled() {
    const char *v = std::getenv("SWB_BATCH_PACK");
    return !(v && v[0] == '0');
}

// Highest H + open a half of a packed lane may reach before its pair is scored
// again in int32; a pair whose best score is bounded by match * n + 256 below
// it is packed without that risk.
constexpr int32_t kSatLimit = 32767 - 256;

// Which packed pairs run on one warp, strip after strip, instead of one strip
// per warp chained through the hand-off buffer.  With far more pairs than
// resident warps a short pair needs no pipeline across warps (whose strips
// would each spin while the strip above gets ahead); a long one keeps it, so
// that no single warp holds the batch's tail.  A pair runs whole when its
// packed rectangle is at most a tenth of one warp's share of the launch's
// cells: on the 100,000-pair batch that is about 8 strips of 448 rows
// (packed kernel 195.4 -> 176.2 ms; whole up to 16 strips, 206.0 ms).
// SWB_BATCH16_WHOLE=k instead runs pairs of at most k strips whole (0: none).
constexpr int64_t kWholeShareDiv = 10;
int32_t packed_whole_strips() {
    if (const char *v = std::getenv("SWB_BATCH16_WHOLE")) return std::max(0, std::atoi(v));
    return -1;
}

// Positions of `order` whose pair may run packed (its best score is bounded
// below the 16-bit limit, or the test flag packs every pair) and the others.
void split_packable(const std::vector<PairInfo> &info, const std::vector<int64_t> &order, const swb_scoring *sc,
                    uint32_t flags, std::vector<int64_t> &ppos, std::vector<int64_t> &rest) {
    for (size_t k = 0; k < order.size(); ++k) {
        const PairInfo &p = info[(size_t)order[k]];
        const bool fits = (int64_t)sc->match * p.n + 256 <= kSatLimit;
        if (fits || (flags & SWB_FLAG_TEST_PACK_ANY)) ppos.push_back((int64_t)k);
        else rest.push_back((int64_t)k);
    }
}

// The host half of a packed pass (see layout_packed).
struct PackedLayout {
    int R = 0;                    // rows per lane it was laid out for (0: none)
    std::vector<int64_t> pos;     // the positions of `order` it covers, as given
    std::vector<PackedPair> pp;   // packed pairs
    std::vector<int2> up;         // work items (packed pair, strip)
    int64_t units = 0, hb = 0;    // strips (best records) and hand-off entries
};

// The host half of the packed pass over the positions `pos` of `order` with R
// rows per lane: pairs sorted by strip count and width and taken two at a time
// (a pair whose neighbour has another strip count gets an empty partner), each
// packed pair whole or chained, and the work items in their claim order.
void layout_packed(swb_ctx *c, const std::vector<PairInfo> &info, const std::vector<int64_t> &order,
                   std::vector<int64_t> pos, uint32_t flags, int R, PackedLayout &L) {
    L.R = R;
    L.pos = pos;
    const int64_t H = 32LL * R;
    const int32_t whole_max = packed_whole_strips();  // -1: by the cell share
    auto strips = [&](int64_t k) { return (info[(size_t)order[(size_t)k]].m + H - 1) / H; };
    // strip count, then width, both descending
    sort_desc(pos, [&](int64_t x) {
        return ((uint64_t)strips(x) << 32) | (uint64_t)info[(size_t)order[(size_t)x]].n;
    });
    const int32_t dummy = (int32_t)order.size();  // slot of an empty half
    std::vector<PackedPair> &pp = L.pp;
    std::vector<int2> &up = L.up;  // work items
    pp.clear();
    up.clear();
    int64_t units = 0, hb = 0;
    for (size_t i = 0; i < pos.size();) {
        const int64_t ka = pos[i];
        const int64_t kb = (i + 1 < pos.size() && strips(pos[i + 1]) == strips(ka)) ? pos[i + 1] : -1;
        i += kb >= 0 ? 2 : 1;
        PackedPair d;
        std::memset(&d, 0, sizeof d);
        const int64_t ks[2] = {ka, kb};
        for (int h = 0; h < 2; ++h) {
            if (ks[h] < 0) {
                d.slot[h] = dummy;
                d.tie[h].mode = kTieRowMajor;
                continue;
            }
            const PairInfo &p = info[(size_t)order[(size_t)ks[h]]];
            d.row_off[h] = p.row_off;
            d.col_off[h] = p.col_off;
            d.m[h] = (int32_t)p.m;
            d.n[h] = (int32_t)p.n;
            d.slot[h] = (int32_t)ks[h];
            int32_t G = 0, T = 0;
            int64_t P1 = 0, P2 = 0;
            const bool refok = reference_geometry(p.m, p.n, &G, &T, &P1, &P2);
            d.tie[h].mode = ((flags & SWB_FLAG_TIE_ROWMAJOR) || !refok) ? kTieRowMajor : kTieReference;
            d.tie[h].G = G;
            d.tie[h].T = T;
            d.tie[h].C = refok ? P2 / G : 1;
        }
        d.M = std::max(d.m[0], d.m[1]);
        d.N = std::max(d.n[0], d.n[1]);
        d.nstrips = (int32_t)((d.M + H - 1) / H);
        d.unit0 = (int32_t)units;
        if (d.nstrips > 1) {
            d.hbuf_off = hb;
            hb += d.N;
        }
        units += d.nstrips;
        pp.push_back(d);
    }
    // whole pairs and the work items (pairs stay in the order above)
    double rect = 0.0;
    for (const PackedPair &d : pp) rect += (double)d.M * (double)d.N;
    const double share = rect / std::max(1, batch16_resident_warps(R, c->sms, c->max_blocks));
    std::vector<int32_t> chained;  // strip counts descending, as pp
    for (size_t q = 0; q < pp.size(); ++q) {
        PackedPair &d = pp[q];
        d.whole = whole_max >= 0 ? (d.nstrips <= whole_max ? 1 : 0)
                                 : ((double)d.M * (double)d.N * (double)kWholeShareDiv <= share ? 1 : 0);
        if (!d.whole) chained.push_back((int32_t)q);
    }
    // Claim order.  A chained pair's strip s waits until strip s - 1 is about
    // kLagSteps steps ahead; claimed pair by pair, the warps that take strips
    // 0..s of a pair start together and strip s spins s times that long (16% of
    // the packed pass on the 100,000-pair batch).  So the chained pairs go
    // strip-major (strip 0 of each, then strip 1, ...), and each strip is
    // claimed long after the one above it.  A pair whose own chain (N columns
    // plus the lag of every strip) is at least half of one warp's share of the
    // launch would then finish late and hold the tail: those go first, pair by
    // pair.  Whole pairs follow, largest first, and fill the tail.  Every strip
    // is claimed after the strip it waits for.
    constexpr double kLagSteps = 84.0;
    const double share_steps = share / (double)H;
    std::vector<int32_t> flow;  // non-critical chained pairs, strip counts descending
    for (int32_t q : chained) {
        const PackedPair &d = pp[(size_t)q];
        if (2.0 * ((double)d.N + (d.nstrips - 1) * kLagSteps) >= share_steps)
            for (int32_t s = 0; s < d.nstrips; ++s) up.push_back(make_int2(q, s));
        else
            flow.push_back(q);
    }
    // (pp is sorted by strip count, so the pairs of `flow` with more than s
    // strips are a prefix of it)
    for (int32_t s = 0; !flow.empty() && s < pp[(size_t)flow[0]].nstrips; ++s)
        for (size_t i = 0; i < flow.size() && pp[(size_t)flow[i]].nstrips > s; ++i)
            up.push_back(make_int2(flow[i], s));
    for (size_t q = 0; q < pp.size(); ++q)
        if (pp[q].whole) up.push_back(make_int2((int32_t)q, 0));
    L.units = units;
    L.hb = hb;
}

// The packed scoring pass over the positions `pos` of `order` with R rows per
// lane (the layout `pre` when it was made for the same R and positions).  Fills
// pbest[k] for every k in pos and appends to `redo` the positions whose pair
// reached the 16-bit limit.
int run_packed(swb_ctx *c, const BatchArgs &base, const std::vector<PairInfo> &info,
               const std::vector<int64_t> &order, const std::vector<int64_t> &pos, uint32_t flags, int R,
               std::vector<BestRec> &pbest, std::vector<int64_t> &redo, float *ms,
               const PackedLayout *pre = nullptr) {
    cudaError_t e;
    PackedLayout local;
    const PackedLayout *L = pre;
    if (!L || L->R != R || L->pos != pos) {
        layout_packed(c, info, order, pos, flags, R, local);
        L = &local;
    }
    const std::vector<PackedPair> &pp = L->pp;
    const std::vector<int2> &up = L->up;
    const int64_t units = L->units, hb = L->hb;
    const int64_t np = (int64_t)pp.size(), nslots = (int64_t)order.size() + 1, items = (int64_t)up.size();
    const size_t pp_bytes = sizeof(PackedPair) * (size_t)np, up_bytes = sizeof(int2) * (size_t)items;
    const size_t back = sizeof(BestRec) * (size_t)nslots + sizeof(int32_t) * (size_t)nslots + 64;
    if ((e = c->b_pairs.ensure(pp_bytes)) != cudaSuccess || (e = c->b_units.ensure(up_bytes)) != cudaSuccess ||
        (e = c->b_hbuf.ensure(sizeof(int4) * (size_t)std::max<int64_t>(1, hb))) != cudaSuccess ||
        (e = c->b_gbest.ensure(sizeof(int32_t) * (size_t)nslots)) != cudaSuccess ||
        (e = c->b_ubest.ensure(2 * sizeof(BestRec) * (size_t)std::max<int64_t>(1, units))) != cudaSuccess ||
        (e = c->b_pbest.ensure(sizeof(BestRec) * (size_t)nslots)) != cudaSuccess ||
        (e = c->b_sat.ensure(sizeof(int32_t) * (size_t)nslots)) != cudaSuccess ||
        (e = c->b_ctl.ensure(4 * sizeof(int32_t))) != cudaSuccess ||
        (e = c->h_stage.ensure(std::max(pp_bytes + up_bytes, back) + 64)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "packed batch buffers");
    uint8_t *hs = (uint8_t *)c->h_stage.p;
    std::memcpy(hs, pp.data(), pp_bytes);
    std::memcpy(hs + pp_bytes, up.data(), up_bytes);
    Batch16Args a{};
    a.rcode = base.rcode;
    a.ctab = base.ctab;
    a.open = base.open;
    a.open2 = (uint32_t)(uint16_t)(int16_t)base.open * 0x00010001u;
    a.ext2 = (uint32_t)(uint16_t)(int16_t)base.ext * 0x00010001u;
    a.gx2 = (uint32_t)(uint16_t)(int16_t)base.gx * 0x00010001u;
    a.mm4 = base.tab_hi;
    a.sat_lim = kSatLimit;
    a.pairs = (const PackedPair *)c->b_pairs.p;
    a.items = (const int2 *)c->b_units.p;
    a.nunits = items;
    a.hbuf = (int4 *)c->b_hbuf.p;
    a.gbest = (int32_t *)c->b_gbest.p;
    a.ubest = (BestRec *)c->b_ubest.p;
    a.ctl = (int32_t *)c->b_ctl.p;
    a.sat = (int32_t *)c->b_sat.p;
    a.wait_limit = c->wait_cycles;
    if ((e = cudaMemcpyAsync(c->b_pairs.p, hs, pp_bytes, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(c->b_units.p, hs + pp_bytes, up_bytes, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
        (hb > 0 && (e = cudaMemsetAsync(a.hbuf, 0xFF, sizeof(int4) * (size_t)hb, c->stream)) != cudaSuccess) ||
        (e = cudaMemsetAsync(a.gbest, 0, sizeof(int32_t) * (size_t)nslots, c->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(c->b_pbest.p, 0, sizeof(BestRec) * (size_t)nslots, c->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(a.sat, 0, sizeof(int32_t) * (size_t)nslots, c->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(a.ctl, 0, 4 * sizeof(int32_t), c->stream)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "packed batch set-up");
    cudaEventRecord(c->ev0, c->stream);
    if ((e = batch16_launch(a, R, c->sms, c->max_blocks, np, (BestRec *)c->b_pbest.p, c->stream)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "packed batch launch");
    cudaEventRecord(c->ev1, c->stream);
    BestRec *hb_best = (BestRec *)hs;
    int32_t *hsat = (int32_t *)(hs + sizeof(BestRec) * (size_t)nslots);
    int32_t *hctl = hsat + nslots;
    if ((e = cudaMemcpyAsync(hb_best, c->b_pbest.p, sizeof(BestRec) * (size_t)nslots, cudaMemcpyDeviceToHost,
                             c->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(hsat, a.sat, sizeof(int32_t) * (size_t)nslots, cudaMemcpyDeviceToHost, c->stream)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(hctl, a.ctl, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c->stream)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "packed batch");
    if (hctl[1] != 0) return ctx_fail(c, SWB_ETIMEOUT, "batch: a bounded wait between strips ran out");
    for (int64_t k : pos) {
        if (hsat[k]) redo.push_back(k);
        else pbest[(size_t)k] = hb_best[k];
    }
    float t = 0.f;
    cudaEventElapsedTime(&t, c->ev0, c->ev1);
    if (ms) *ms += t;
    return SWB_OK;
}

// Packed batches at least this large may probe the candidates on their own pairs.
constexpr int64_t kTuneMinPairs = 16384;

// Rows per lane of the packed pass over `ppos`: SWB_BATCH16_R (8 or 14), else
// the autotuner's recorded choice for the batch's bucket, else timed probes:
// candidate i scores the pairs at indices i, i + 8, i + 16, ... of ppos (an
// eighth of the batch each, the same length mix), those results are kept and
// their positions leave ppos, and the candidate with the most cells per ms is
// recorded.  Batches below kTuneMinPairs take kBatch16R.
// Rows per lane of the packed pass over ppos when no probe is needed:
// SWB_BATCH16_R, the recorded choice of the batch's bucket, or kBatch16R for
// batches too small to probe; 0 when the bucket is new and the batch large.
int packed_rows_known(swb_ctx *c, const std::vector<PairInfo> &info, const std::vector<int64_t> &order,
                      const std::vector<int64_t> &ppos, const char **how, std::string *key_out) {
    if (const char *v = std::getenv("SWB_BATCH16_R")) {
        const int r = std::atoi(v);
        if (r == kBatch16R || r == kBatch16RShort) {
            *how = "SWB_BATCH16_R";
            return r;
        }
    }
    *how = "default";
    if (ppos.empty()) return kBatch16R;
    // ceil(log2) of the cells-weighted median rows and columns of the packed
    // pairs: the median's power-of-two bucket, from per-bucket cell sums
    auto median = [&](bool rows) {
        double w[64] = {0.0}, total = 0.0;
        for (int64_t k : ppos) {
            const PairInfo &p = info[(size_t)order[(size_t)k]];
            const int64_t x = rows ? p.m : p.n;
            int b = 0;
            while (b < 62 && (1LL << b) < x) ++b;
            const double cells = (double)p.m * (double)p.n;
            w[b] += cells;
            total += cells;
        }
        double acc = 0.0;
        for (int b = 0; b < 64; ++b)
            if ((acc += w[b]) >= 0.5 * total) return (int64_t)1 << b;
        return (int64_t)1 << 62;
    };
    const std::string key = batch_tune_key(c->sms, "batch16", median(true), median(false));
    if (key_out) *key_out = key;
    int cached = 0;
    if (tune_lookup(key, &cached) && (cached == kBatch16R || cached == kBatch16RShort)) {
        *how = "cached";
        return cached;
    }
    return (int64_t)ppos.size() < kTuneMinPairs ? kBatch16R : 0;
}

int tune_packed(swb_ctx *c, const BatchArgs &base, const std::vector<PairInfo> &info,
                const std::vector<int64_t> &order, std::vector<int64_t> &ppos, uint32_t flags,
                std::vector<BestRec> &pbest, std::vector<int64_t> &redo, float *ms, int32_t *launches, int *R,
                const char **how) {
    std::string key;
    const int known = packed_rows_known(c, info, order, ppos, how, &key);
    *R = known > 0 ? known : kBatch16R;
    if (known > 0) return SWB_OK;
    const int cands[2] = {kBatch16R, kBatch16RShort};
    double rate[2] = {0.0, 0.0};
    for (int i = 0; i < 2; ++i) {
        std::vector<int64_t> sample;
        double cells = 0.0;
        for (size_t q = (size_t)i; q < ppos.size(); q += 8) {
            sample.push_back(ppos[q]);
            const PairInfo &p = info[(size_t)order[(size_t)ppos[q]]];
            cells += (double)p.m * (double)p.n;
        }
        float t = 0.f;
        const int rc = run_packed(c, base, info, order, sample, flags, cands[i], pbest, redo, &t);
        if (rc != SWB_OK) return rc;
        *launches += 2;
        if (ms) *ms += t;
        rate[i] = t > 0.f ? cells / (double)t : 0.0;
    }
    std::vector<int64_t> rest;
    rest.reserve(ppos.size());
    for (size_t q = 0; q < ppos.size(); ++q)
        if (q % 8 >= 2) rest.push_back(ppos[q]);
    ppos.swap(rest);
    *R = rate[1] > rate[0] ? cands[1] : cands[0];
    *how = "probed";
    tune_record(key, *R);
    return SWB_OK;
}

// Host phases of a batched call on stderr (options.verbose bit 0): the time
// since the previous mark, in ms.
struct PhaseLog {
    bool on;
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    explicit PhaseLog(const swb_ctx *c) : on(c && (c->opts.verbose & 1)) {}
    void mark(const char *what) {
        if (!on) return;
        const auto now = std::chrono::steady_clock::now();
        std::fprintf(stderr, "swb batch: %-22s %9.3f ms\n", what,
                     std::chrono::duration<double, std::milli>(now - t).count());
        t = now;
    }
};

size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }

size_t pow2_at_least(size_t x) {
    size_t p = 1 << 16;
    while (p < x) p <<= 1;
    return p;
}

// The instantiated graph for a shape (traced or not, rows per lane, grid cap,
// size class: grids sized for at most 2^size_class work units and pairs),
// captured on first use.  Its kernels read the call header at c->g_hdr.p, so the
// graph never changes for a shape; the scoring kernels' parameters are set per
// replay (graph_set_scoring).
cudaError_t graph_for(swb_ctx *c, bool traced, int R, int cap, int size_class, swb_ctx::GraphEntry **out) {
    for (auto &g : c->graphs)
        if (g.exec && g.traced == (int)traced && g.R == R && g.cap == cap && g.size_class == size_class) {
            *out = &g;
            return cudaSuccess;
        }
    const int64_t max_units = 1LL << size_class;
    cudaError_t e;
    if (!c->cap_stream && (e = cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return e;
    const GraphHdr *h = (const GraphHdr *)c->g_hdr.p;
    if ((e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return e;
    cudaError_t q = cudaEventRecordWithFlags(c->ev0, c->cap_stream, cudaEventRecordExternal);
    if (q == cudaSuccess) q = batch_graph_enqueue(h, traced, R, c->sms, cap, max_units, c->ev1, c->cap_stream);
    if (q == cudaSuccess && traced) q = tb::walk_graph_enqueue(h, c->sms, max_units, c->cap_stream);
    if (q == cudaSuccess && traced) q = cudaEventRecordWithFlags(c->ev2, c->cap_stream, cudaEventRecordExternal);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(c->cap_stream, &graph);
    if (q != cudaSuccess) e = q;
    // the scoring kernels' nodes
    cudaGraphNode_t scoring[2] = {nullptr, nullptr};
    cudaKernelNodeParams skp[2] = {};
    if (e == cudaSuccess) {
        const void *f[2];
        batch_graph_scoring_funcs(traced, R, f);
        size_t nn = 0;
        e = cudaGraphGetNodes(graph, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        if (e == cudaSuccess && nn > 0) e = cudaGraphGetNodes(graph, nodes.data(), &nn);
        for (size_t i = 0; e == cudaSuccess && i < nn; ++i) {
            cudaGraphNodeType t;
            if ((e = cudaGraphNodeGetType(nodes[i], &t)) != cudaSuccess || t != cudaGraphNodeTypeKernel) continue;
            cudaKernelNodeParams kp{};
            if ((e = cudaGraphKernelNodeGetParams(nodes[i], &kp)) != cudaSuccess) break;
            for (int k = 0; k < 2; ++k)
                if (kp.func == f[k]) {
                    scoring[k] = nodes[i];
                    skp[k] = kp;
                }
        }
        if (e == cudaSuccess && (!scoring[0] || !scoring[1])) e = cudaErrorInvalidValue;
    }
    cudaGraphExec_t x = nullptr;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&x, graph, 0);
    if (e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return e;
    }
    swb_ctx::GraphEntry *slot = nullptr;
    for (auto &g : c->graphs)
        if (!g.exec) {
            slot = &g;
            break;
        }
    if (!slot) {
        slot = &c->graphs[c->graph_next];
        c->graph_next = (c->graph_next + 1) % (int)(sizeof c->graphs / sizeof c->graphs[0]);
        cudaGraphExecDestroy(slot->exec);
        cudaGraphDestroy(slot->graph);
    }
    slot->graph = graph;
    slot->exec = x;
    for (int k = 0; k < 2; ++k) {
        slot->scoring[k] = scoring[k];
        slot->kp[k] = skp[k];
        slot->kp[k].kernelParams = nullptr;
        slot->kp[k].extra = nullptr;
    }
    slot->args_valid = false;
    slot->traced = traced;
    slot->R = R;
    slot->cap = cap;
    slot->size_class = size_class;
    *out = slot;
    return cudaSuccess;
}

// Sets this replay's BatchArgs (and the header address) on the graph's two
// scoring kernels, unless the ones set last time are the same (the serving
// loop's steady state: same scoring, same buffers).
cudaError_t graph_set_scoring(swb_ctx *c, swb_ctx::GraphEntry *g, const BatchArgs &ba) {
    static_assert(sizeof(BatchArgs) <= sizeof g->set_args, "BatchArgs cache");
    if (g->args_valid && std::memcmp(g->set_args, &ba, sizeof ba) == 0) return cudaSuccess;
    const GraphHdr *h = (const GraphHdr *)c->g_hdr.p;
    BatchArgs a = ba;
    void *args[] = {&a, &h};
    for (int k = 0; k < 2; ++k) {
        cudaKernelNodeParams kp = g->kp[k];
        kp.kernelParams = args;
        const cudaError_t e = cudaGraphExecKernelNodeSetParams(g->exec, g->scoring[k], &kp);
        if (e != cudaSuccess) {
            g->args_valid = false;
            return e;
        }
    }
    std::memcpy(g->set_args, &ba, sizeof ba);
    g->args_valid = true;
    return cudaSuccess;
}

// Results of a graphed pass, per entry k of bp (pair order[k]).
struct GraphPass {
    std::vector<BatchPair> bp;
    std::vector<BestRec> pbest;
    bool tab = false;
    const uint8_t *d_seq = nullptr;
    const uint8_t *rcode = nullptr;
    const uint32_t *ctab = nullptr;
    float ms1 = 0.f, ms2 = 0.f;
    // traced passes: walker state, reversed ops and crosspoints (pinned host copies)
    const int64_t *states = nullptr;
    const char *ops = nullptr;
    const int64_t *xps = nullptr;
    std::vector<int64_t> ops_off, xp_off, ops_cap, xp_cap;
};

// One graphed pass over the active pairs `order` of a host batch: the sequences
// and every descriptor go to the device in one copy, one graph replay scores
// every pair (traced: keeping the stores and walking every pair with a positive
// score), and one copy brings the results back.
int graph_pass(swb_ctx *c, const uint8_t *h_seq, int64_t seq_bytes, const std::vector<PairInfo> &info,
               const std::vector<int64_t> &order, const swb_scoring *sc, uint32_t flags, bool traced,
               swb_batch_result *out, GraphPass &gp) {
    cudaError_t e;
    PhaseLog ph(c);
    const int R = traced ? kBatchR : batch_score_rows_per_lane();
    std::vector<int32_t> unit_pair;
    int64_t hb = 0, srn = 0, scn = 0, ops_total = 0, xp_total = 0;
    layout_units(info, order, flags, 32 * R, gp.bp, unit_pair, &hb);
    ph.mark("graph: layout units");
    const int64_t np = (int64_t)gp.bp.size(), nu = (int64_t)unit_pair.size();
    const int kS = tb::state_slots();
    if (traced) {
        layout_stores(gp.bp, out->items, order, &srn, &scn, &ops_total, &xp_total);
        if ((uint64_t)(srn + scn) * sizeof(int2) > c->opts.hbm_budget_bytes)
            return ctx_fail(c, SWB_ENOMEM_BUDGET, "traced pairs' special rows and columns exceed the HBM budget");
        gp.ops_off.resize((size_t)np);
        gp.xp_off.resize((size_t)np);
        gp.ops_cap.resize((size_t)np);
        gp.xp_cap.resize((size_t)np);
        int64_t oo = 0, xo = 0;
        for (int64_t k = 0; k < np; ++k) {
            const BatchPair &d = gp.bp[(size_t)k];
            gp.ops_off[(size_t)k] = oo;
            gp.xp_off[(size_t)k] = xo;
            gp.ops_cap[(size_t)k] = (int64_t)d.m + d.n + 8;
            gp.xp_cap[(size_t)k] = d.m / out->items[order[(size_t)k]].xpoint_interval + 8;
            oo += gp.ops_cap[(size_t)k];
            xo += gp.xp_cap[(size_t)k];
        }
        ops_total = oo;
        xp_total = xo;
    }
    // device layouts (16-byte aligned sections)
    const size_t wa_bytes = tb::walk_args_bytes();
    const size_t in_pairs = 0, in_units = al16(in_pairs + sizeof(BatchPair) * (size_t)np);
    const size_t in_walk = al16(in_units + sizeof(int32_t) * (size_t)nu);
    const size_t in_seq = al16(in_walk + (traced ? wa_bytes * (size_t)np : 0));
    const size_t in_bytes = al16(in_seq + (size_t)seq_bytes + 64);
    const size_t w_hbuf = 0, w_gbest = al16(w_hbuf + sizeof(int4) * (size_t)hb);
    const size_t w_ubest = al16(w_gbest + sizeof(int32_t) * (size_t)np);
    const size_t w_rcode = al16(w_ubest + sizeof(BestRec) * (size_t)nu);
    const size_t w_ctab = al16(w_rcode + (size_t)seq_bytes + 64);
    const size_t w_srows = al16(w_ctab + sizeof(uint32_t) * ((size_t)seq_bytes + 64));
    const size_t w_scols = al16(w_srows + sizeof(int2) * (size_t)srn);
    const size_t work_bytes = al16(w_scols + sizeof(int2) * (size_t)scn);
    const size_t o_ctl = 0, o_pbest = 32;
    const size_t o_states = al16(o_pbest + sizeof(BestRec) * (size_t)np);
    const size_t o_xps = al16(o_states + (traced ? sizeof(int64_t) * (size_t)kS * (size_t)np : 0));
    const size_t o_ops = al16(o_xps + sizeof(int64_t) * 4 * (size_t)xp_total);
    const size_t out_bytes = al16(o_ops + (size_t)ops_total);
    const size_t hdr_bytes = al16(sizeof(GraphHdr)), hdr_all = hdr_bytes + 256 + 32;
    const bool fresh_hdr = c->g_hdr.p == nullptr;
    if ((e = c->g_hdr.ensure(hdr_all)) != cudaSuccess || (e = c->g_in.ensure(in_bytes)) != cudaSuccess ||
        (e = c->g_work.ensure(work_bytes)) != cudaSuccess || (e = c->g_out.ensure(out_bytes)) != cudaSuccess ||
        (traced && (e = c->g_dir.ensure(tb::walk_batch_dir_bytes(c->sms, tb::walk_graph_ctas(c->sms)))) != cudaSuccess) ||
        (e = c->h_gin.ensure(pow2_at_least(hdr_bytes + in_bytes))) != cudaSuccess ||
        (e = c->h_gout.ensure(pow2_at_least(out_bytes))) != cudaSuccess)
        return ctx_cuda_fail(c, e, "graphed batch buffers");
    uint8_t *dh = (uint8_t *)c->g_hdr.p, *din = (uint8_t *)c->g_in.p, *dw = (uint8_t *)c->g_work.p,
            *dout = (uint8_t *)c->g_out.p;
    if (fresh_hdr && (e = cudaMemsetAsync(dh, 0, hdr_all, c->stream)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "graphed batch header");
    // the header
    uint8_t *hs = (uint8_t *)c->h_gin.p;
    GraphHdr g{};
    g.ba.open = sc->gap_open;
    g.ba.ext = sc->gap_extend;
    g.ba.gx = std::max(sc->gap_open, sc->gap_extend);
    g.ba.mt1 = sc->match - sc->gap_open;
    g.ba.mm1 = sc->mismatch - sc->gap_open;
    const uint32_t mmb = (uint32_t)(uint8_t)(int8_t)g.ba.mm1;
    g.ba.tab_hi = mmb * 0x01010101u;
    g.x1 = ((uint32_t)(uint8_t)(int8_t)g.ba.mt1 ^ mmb) & 0xFFu;
    g.tab_ok = (g.ba.mt1 >= -128 && g.ba.mt1 <= 127 && g.ba.mm1 >= -128 && g.ba.mm1 <= 127) ? 1 : 0;
    g.ba.seq = din + in_seq;
    g.ba.cseq = din + in_seq;
    g.ba.rcode = dw + w_rcode;
    g.ba.ctab = (const uint32_t *)(dw + w_ctab);
    g.ba.pairs = (const BatchPair *)(din + in_pairs);
    g.ba.unit_pair = (const int32_t *)(din + in_units);
    g.ba.nunits = 0;  // read from the header (nunits_dev): the graph's parameters stay the same
    g.ba.nunits_dev = reinterpret_cast<const int64_t *>(dh + offsetof(GraphHdr, nunits));
    g.nunits = nu;
    g.ba.hbuf = (int4 *)(dw + w_hbuf);
    g.ba.gbest = (int32_t *)(dw + w_gbest);
    g.ba.ubest = (BestRec *)(dw + w_ubest);
    g.ba.ctl = (int32_t *)(dout + o_ctl);
    g.ba.wait_limit = c->wait_cycles;
    g.ba.srows = traced ? (int2 *)(dw + w_srows) : nullptr;
    g.ba.scols = traced ? (int2 *)(dw + w_scols) : nullptr;
    g.pbest = (BestRec *)(dout + o_pbest);
    g.npairs = np;
    g.seq_bytes = seq_bytes;
    g.hbuf_entries = hb;
    g.walk_args = traced ? (void *)(din + in_walk) : nullptr;
    g.walk_states = traced ? (int64_t *)(dout + o_states) : nullptr;
    g.walk_dir = traced ? (uint32_t *)c->g_dir.p : nullptr;
    g.lut = dh + hdr_bytes;
    g.presence = (uint32_t *)(dh + hdr_bytes + 256);
    g.out = (int32_t *)(dout + o_ctl);
    std::memcpy(hs, &g, sizeof g);
    // the inputs
    uint8_t *hin = hs + hdr_bytes;
    std::memcpy(hin + in_pairs, gp.bp.data(), sizeof(BatchPair) * (size_t)np);
    std::memcpy(hin + in_units, unit_pair.data(), sizeof(int32_t) * (size_t)nu);
    if (traced) {
        std::vector<tb::WalkInputs> win((size_t)np);
        for (int64_t k = 0; k < np; ++k) {
            const BatchPair &d = gp.bp[(size_t)k];
            tb::WalkInputs &w = win[(size_t)k];
            std::memset(&w, 0, sizeof w);
            w.rows = g.ba.seq + d.row_off;
            w.cols = g.ba.seq + d.col_off;
            w.m = d.m;
            w.n = d.n;
            w.sc = *sc;
            w.srows = g.ba.srows + d.sr_off;
            w.scols = g.ba.scols + d.sc_off;
            w.rr1 = d.m;
            w.cc1 = d.n;
            w.xp_interval = out->items[order[(size_t)k]].xpoint_interval;
            w.ops = (char *)(dout + o_ops) + gp.ops_off[(size_t)k];
            w.ops_cap = gp.ops_cap[(size_t)k];
            w.xps = (int64_t *)(dout + o_xps) + 4 * gp.xp_off[(size_t)k];
            w.xp_cap = gp.xp_cap[(size_t)k];
        }
        tb::pack_walk_args(win.data(), np, g.walk_states, hin + in_walk);
    }
    ph.mark("graph: descriptors");
    copy_parallel(hin + in_seq, h_seq, (size_t)seq_bytes);
    ph.mark("graph: sequences staged");
    // size class: the smallest power of two >= the unit count (pairs <= units), up
    // to one that no longer shrinks any grid
    int size_class = 0;
    while ((1LL << size_class) < nu && size_class < 30) ++size_class;
    {
        int full = 0;
        while ((1LL << full) < 64LL * std::max(1, c->sms)) ++full;
        size_class = std::min(size_class, full);
    }
    swb_ctx::GraphEntry *ge = nullptr;
    if ((e = graph_for(c, traced, R, c->max_blocks, size_class, &ge)) != cudaSuccess ||
        (e = graph_set_scoring(c, ge, g.ba)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "batch graph");
    uint8_t *hout = (uint8_t *)c->h_gout.p;
    if ((e = cudaMemcpyAsync(dh, hs, sizeof g, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(din, hin, in_seq + (size_t)seq_bytes, cudaMemcpyHostToDevice, c->stream)) != cudaSuccess ||
        (e = cudaGraphLaunch(ge->exec, c->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(hout, dout, out_bytes, cudaMemcpyDeviceToHost, c->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(c->stream)) != cudaSuccess)
        return ctx_cuda_fail(c, e, "batch graph replay");
    ph.mark("graph: copies + replay");
    const int32_t *ctl = (const int32_t *)(hout + o_ctl);
    if (ctl[1] != 0) return ctx_fail(c, SWB_ETIMEOUT, "batch: a bounded wait between strips ran out");
    gp.tab = ctl[4] != 0;
    gp.d_seq = g.ba.seq;
    gp.rcode = g.ba.rcode;
    gp.ctab = g.ba.ctab;
    gp.pbest.resize((size_t)np);
    std::memcpy(gp.pbest.data(), hout + o_pbest, sizeof(BestRec) * (size_t)np);
    cudaEventElapsedTime(&gp.ms1, c->ev0, c->ev1);
    if (traced) {
        cudaEventElapsedTime(&gp.ms2, c->ev1, c->ev2);
        gp.states = (const int64_t *)(hout + o_states);
        gp.ops = (const char *)(hout + o_ops);
        gp.xps = (const int64_t *)(hout + o_xps);
        for (int64_t k = 0; k < np; ++k) {
            const int64_t *S = gp.states + (size_t)kS * k;
            if (S[tb::slot_err()] != 0 || !S[tb::slot_done()])
                return ctx_fail(c, SWB_ECUDA, "batched walker: inconsistent direction data");
        }
    }
    return SWB_OK;
}

int batch_run(swb_ctx *c, const uint8_t *h_seq, const uint8_t *d_seq_in, int64_t seq_bytes, const swb_pair_ref *pairs,
              int64_t npairs, const swb_scoring *sc, uint32_t flags, double trace_frac, swb_batch_result *out,
              bool stores_first) {
    const auto t0 = std::chrono::steady_clock::now();
    PhaseLog ph(c);
    std::memset(out, 0, sizeof *out);
    if (!sc) return ctx_fail(c, SWB_EINVAL, "scoring is NULL");
    if (sc->match < 1 || sc->mismatch > -1 || sc->gap_open > -1 || sc->gap_extend > -1)
        return ctx_fail(c, SWB_EINVAL, "One or more scoring values were not usable!");
    if (npairs < 0 || (npairs > 0 && !pairs) || seq_bytes < 0 || !(trace_frac >= 0.0 && trace_frac <= 1.0))
        return ctx_fail(c, SWB_EINVAL, "swb_batch_align: bad arguments");
    if (npairs > (int64_t)INT32_MAX / 4) return ctx_fail(c, SWB_EUNSUPPORTED, "too many pairs in one batch");
    // orientation of every pair (src/SWutils.cpp:84-88: the longer one is rows)
    std::vector<PairInfo> info((size_t)npairs);
    int64_t maxlen = 0, cells = 0;
    for (int64_t i = 0; i < npairs; ++i) {
        const swb_pair_ref &r = pairs[i];
        if (r.a_off < 0 || r.a_len < 0 || r.b_off < 0 || r.b_len < 0 || r.a_off > seq_bytes ||
            r.a_len > seq_bytes - r.a_off || r.b_off > seq_bytes || r.b_len > seq_bytes - r.b_off)
            return ctx_fail(c, SWB_EINVAL, "pair %lld: byte range outside the sequence buffer", (long long)i);
        PairInfo &p = info[(size_t)i];
        p.swapped = r.a_len < r.b_len ? 1 : 0;
        p.row_off = p.swapped ? r.b_off : r.a_off;
        p.col_off = p.swapped ? r.a_off : r.b_off;
        p.m = std::max(r.a_len, r.b_len);
        p.n = std::min(r.a_len, r.b_len);
        if (p.m > (int64_t)INT32_MAX - 64) return ctx_fail(c, SWB_EUNSUPPORTED, "sequence longer than 2^31 - 64");
        maxlen = std::max(maxlen, p.m + p.n);
        cells += p.m * p.n;
    }
    {
        const long double worst = (long double)std::max(std::max(sc->match, -sc->mismatch),
                                                        std::max(-sc->gap_open, -sc->gap_extend)) *
                                  (long double)(maxlen + 2);
        if (worst > 2.0e9L) return ctx_fail(c, SWB_EUNSUPPORTED, "scores would leave the int32 range");
    }
    out->npairs = npairs;
    out->cells = cells;
    out->items = (swb_batch_item *)std::calloc((size_t)std::max<int64_t>(1, npairs), sizeof(swb_batch_item));
    if (!out->items) return ctx_fail(c, SWB_ENOMEM, "out of host memory");
    for (int64_t i = 0; i < npairs; ++i) out->items[i].swapped = info[(size_t)i].swapped;

    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
    cudaError_t e;
    // active pairs (both sequences non-empty), longest first (ties: lower index)
    std::vector<int64_t> order;
    order.reserve((size_t)npairs);
    for (int64_t i = 0; i < npairs; ++i)
        if (info[(size_t)i].n > 0) order.push_back(i);
    sort_desc(order, [&](int64_t x) { return (uint64_t)(info[(size_t)x].m * info[(size_t)x].n); });
    for (int64_t i = 0; i < npairs; ++i) {
        int32_t G = 0, T = 0;
        int64_t P1 = 0, P2 = 0;
        reference_geometry(info[(size_t)i].m, info[(size_t)i].n, &G, &T, &P1, &P2);
        out->items[i].xpoint_interval = T > 0 ? 4 * T : 20;
    }
    // host batches run as one replayed graph (sequences and descriptors in one
    // copy, results in one copy); device batches and the store pass of a
    // partially traced batch launch their kernels directly
    // large score-only batches take the packed 16-bit pass (direct launches); the
    // rest of host batches run as one replayed graph
    const int32_t mt1 = sc->match - sc->gap_open, mm1 = sc->mismatch - sc->gap_open;
    const bool pack_candidate = !stores_first && (int64_t)order.size() >= kPackMinPairs && packing_enabled() &&
                                mt1 >= -128 && mt1 <= 127 && mm1 >= -128 && mm1 <= 127;
    const bool use_graph = h_seq != nullptr && !order.empty() && graphs_enabled() && !pack_candidate;
    GraphPass gp;
    ph.mark("orient + order");
    if (use_graph) {
        int rc = graph_pass(c, h_seq, seq_bytes, info, order, sc, flags, stores_first, out, gp);
        if (rc != SWB_OK) return rc;
    }

    const uint8_t *d_seq = d_seq_in;
    if (h_seq && !use_graph) {
        // through the context's pinned staging, copied in by several threads
        if ((e = c->b_seq.ensure((size_t)seq_bytes + 64)) != cudaSuccess ||
            (e = cudaStreamSynchronize(c->stream)) != cudaSuccess ||
            (e = c->h_io.ensure((size_t)std::max<int64_t>(1, seq_bytes))) != cudaSuccess)
            return ctx_cuda_fail(c, e, "batch sequences");
        copy_parallel((uint8_t *)c->h_io.p, h_seq, (size_t)seq_bytes);
        if (seq_bytes > 0 &&
            (e = cudaMemcpyAsync(c->b_seq.p, c->h_io.p, (size_t)seq_bytes, cudaMemcpyHostToDevice, c->stream)) !=
                cudaSuccess)
            return ctx_cuda_fail(c, e, "copy batch sequences");
        d_seq = (const uint8_t *)c->b_seq.p;
        ph.mark("sequences to the device");
    }

    // The packed pass's host layout (sorting, packing, claim order: several ms
    // for 100,000 pairs) is built now, while the sequences are still on their
    // way to the device, whenever its strip height needs no probe.  If the
    // batch then turns out not to be in the table mode, it goes unused.
    PackedLayout early;
    if (pack_candidate && !order.empty() && !use_graph) {
        std::vector<int64_t> ppos, rest;
        split_packable(info, order, sc, flags, ppos, rest);
        const char *how = "";
        const int R = packed_rows_known(c, info, order, ppos, &how, nullptr);
        if (R > 0 && !ppos.empty()) layout_packed(c, info, order, ppos, flags, R, early);
        ph.mark("packed layout");
    }

    BatchArgs base{};
    base.wait_limit = c->wait_cycles;
    base.open = sc->gap_open;
    base.ext = sc->gap_extend;
    base.gx = std::max(sc->gap_open, sc->gap_extend);
    base.mt1 = sc->match - sc->gap_open;
    base.mm1 = sc->mismatch - sc->gap_open;
    bool tab = false;
    int32_t launches = 0;
    if (use_graph) {
        d_seq = gp.d_seq;
        tab = gp.tab;
        if (tab) {
            base.rcode = gp.rcode;
            base.ctab = gp.ctab;
            base.tab_hi = (uint32_t)(uint8_t)(int8_t)base.mm1 * 0x01010101u;
        }
        launches += stores_first ? 8 : 6;
    } else if (!order.empty() && base.mt1 >= -128 && base.mt1 <= 127 && base.mm1 >= -128 && base.mm1 <= 127) {
        // TAB mode when the whole buffer holds at most four distinct bytes
        uint32_t present[256];
        if ((e = c->flags.ensure(256 * sizeof(uint32_t))) != cudaSuccess ||
            (e = stage1_presence(d_seq, seq_bytes, (uint32_t *)c->flags.p, c->stream)) != cudaSuccess ||
            (e = ctx_get(c, present, c->flags.p, sizeof present)) != cudaSuccess)
            return ctx_cuda_fail(c, e, "batch alphabet");
        launches += 1;
        uint8_t lut[256];
        int K = 0;
        for (int i = 0; i < 256; ++i) lut[i] = present[i] ? (uint8_t)(K++) : 7;
        if (K <= 4) {
            tab = true;
            if ((e = c->lut.ensure(256)) != cudaSuccess || (e = c->b_rcode.ensure((size_t)seq_bytes + 64)) != cudaSuccess ||
                (e = c->b_ctab.ensure(sizeof(uint32_t) * ((size_t)seq_bytes + 64))) != cudaSuccess ||
                (e = ctx_put(c, c->lut.p, lut, 256)) != cudaSuccess ||
                (e = batch_encode(d_seq, seq_bytes, (const uint8_t *)c->lut.p, (uint8_t *)c->b_rcode.p,
                                  (uint32_t *)c->b_ctab.p, base.mt1, base.mm1, &base.tab_hi, c->stream)) != cudaSuccess)
                return ctx_cuda_fail(c, e, "batch encode");
            launches += 1;
            base.rcode = (const uint8_t *)c->b_rcode.p;
            base.ctab = (const uint32_t *)c->b_ctab.p;
        }
    }

    auto ensure_stores = [&](int64_t srn, int64_t scn) -> int {
        if ((uint64_t)(srn + scn) * sizeof(int2) > c->opts.hbm_budget_bytes)
            return ctx_fail(c, SWB_ENOMEM_BUDGET, "traced pairs' special rows and columns exceed the HBM budget");
        if ((e = c->b_srows.ensure(sizeof(int2) * (size_t)std::max<int64_t>(1, srn))) != cudaSuccess ||
            (e = c->b_scols.ensure(sizeof(int2) * (size_t)std::max<int64_t>(1, scn))) != cudaSuccess)
            return ctx_cuda_fail(c, e, "batch special rows and columns");
        return SWB_OK;
    };

    // scoring launch (with the stores of every pair when all are traced anyway)
    std::vector<BatchPair> bp;
    std::vector<int32_t> unit_pair;
    std::vector<BestRec> pbest;
    int64_t hb = 0, srn = 0, scn = 0, ops_total = 0, xp_total = 0;
    float ms1 = 0.f;
    const bool first_stores = stores_first && !order.empty();
    const int R1 = first_stores ? kBatchR : batch_score_rows_per_lane();
    if (use_graph) {
        bp = gp.bp;
        pbest = gp.pbest;
        ms1 = gp.ms1;
    } else if (!(pack_candidate && tab)) {
        layout_units(info, order, flags, 32 * R1, bp, unit_pair, &hb);
    }
    if (!order.empty() && !use_graph && pack_candidate && tab) {
        // pairs whose best score is bounded below the 16-bit limit run packed two
        // per warp; the others, and any pair that reached the limit, in int32
        std::vector<int64_t> ppos, rest;
        split_packable(info, order, sc, flags, ppos, rest);
        pbest.assign(order.size(), BestRec{});
        int Rp = kBatch16R;
        const char *how = "";
        int rc = tune_packed(c, base, info, order, ppos, flags, pbest, rest, &ms1, &launches, &Rp, &how);
        if (rc != SWB_OK) return rc;
        if (ph.on) std::fprintf(stderr, "swb batch: packed rows per lane %d (%s)\n", Rp, how);
        if (!ppos.empty()) {
            rc = run_packed(c, base, info, order, ppos, flags, Rp, pbest, rest, &ms1, &early);
            if (rc != SWB_OK) return rc;
            launches += 2;
        }
        ph.mark("packed pass");
        if (!rest.empty()) {
            std::vector<int64_t> sub(rest.size());
            for (size_t i = 0; i < rest.size(); ++i) sub[i] = order[(size_t)rest[i]];
            std::vector<BatchPair> bp2;
            std::vector<int32_t> up2;
            std::vector<BestRec> pb2;
            int64_t hb2 = 0;
            layout_units(info, sub, flags, 32 * R1, bp2, up2, &hb2);
            rc = run_launch(c, d_seq, tab, base, bp2, up2, hb2, false, R1, pb2, &ms1, true);
            if (rc != SWB_OK) return rc;
            launches += 2;
            for (size_t i = 0; i < rest.size(); ++i) pbest[(size_t)rest[i]] = pb2[i];
        }
    } else if (!order.empty() && !use_graph) {
        BatchArgs a1 = base;
        if (first_stores) {
            layout_stores(bp, out->items, order, &srn, &scn, &ops_total, &xp_total);
            int rc = ensure_stores(srn, scn);
            if (rc != SWB_OK) return rc;
            a1.srows = (int2 *)c->b_srows.p;
            a1.scols = (int2 *)c->b_scols.p;
        }
        int rc = run_launch(c, d_seq, tab, a1, bp, unit_pair, hb, first_stores, R1, pbest, &ms1, true);
        if (rc != SWB_OK) return rc;
        launches += 2;
    }
    for (size_t k = 0; k < order.size(); ++k) {
        swb_batch_item &it = out->items[order[k]];
        const BestRec &b = pbest[k];
        if (b.valid) {
            it.score = b.ho - sc->gap_open;
            it.end_row = b.row;
            it.end_col = b.col;
        }
    }
    for (int64_t i = 0; i < npairs; ++i) {
        out->items[i].start_row = out->items[i].end_row;
        out->items[i].start_col = out->items[i].end_col;
    }
    out->stage1_ms = ms1;
    ph.mark("scoring pass");

    // traceback of the best-scoring pairs
    const int64_t ntrace =
        stores_first ? npairs : std::min<int64_t>(npairs, (int64_t)std::ceil(trace_frac * (double)npairs - 1e-9));
    if (ntrace > 0) {
        const auto t1 = std::chrono::steady_clock::now();
        // the ntrace best scores (ties: lower index first)
        std::vector<int64_t> byscore((size_t)npairs);
        std::iota(byscore.begin(), byscore.end(), 0);
        std::partial_sort(byscore.begin(), byscore.begin() + ntrace, byscore.end(), [&](int64_t x, int64_t y) {
            const int32_t sx = out->items[x].score, sy = out->items[y].score;
            return sx != sy ? sx > sy : x < y;
        });
        byscore.resize((size_t)ntrace);
        std::sort(byscore.begin(), byscore.end());
        std::vector<int64_t> tr;  // traced pairs that have an alignment (score > 0)
        for (int64_t i : byscore) {
            out->items[i].traced = 1;
            if (out->items[i].score > 0) tr.push_back(i);
        }
        out->n_traced = ntrace;
        // the layout whose special rows and columns the walker reads, per traced pair
        std::vector<BatchPair> bpw(tr.size());
        ph.mark("select traced pairs");
        if (first_stores) {
            std::vector<int64_t> pos((size_t)npairs, -1);
            for (size_t k = 0; k < order.size(); ++k) pos[(size_t)order[k]] = (int64_t)k;
            for (size_t k = 0; k < tr.size(); ++k) bpw[k] = bp[(size_t)pos[(size_t)tr[k]]];
        } else if (!tr.empty()) {
            // store pass over the traced pairs: special rows every 512 rows (every
            // strip), special columns every 256 columns.  The path ends at the end
            // cell, and no cell below or right of it feeds a cell above and left
            // of it, so only rows 0..end_row and columns 0..end_col are computed
            // (their values and the best cell's tie key are the whole pair's).
            std::vector<int32_t> up2;
            int64_t hb2 = 0;
            std::vector<std::pair<int64_t, int64_t>> ext(tr.size());
            for (size_t k = 0; k < tr.size(); ++k)
                ext[k] = {out->items[tr[k]].end_row + 1, out->items[tr[k]].end_col + 1};
            layout_units(info, tr, flags, kBatchStripRows, bpw, up2, &hb2, &ext);
            layout_stores(bpw, out->items, tr, &srn, &scn, &ops_total, &xp_total);
            int rc = ensure_stores(srn, scn);
            if (rc != SWB_OK) return rc;
            BatchArgs b2 = base;
            b2.srows = (int2 *)c->b_srows.p;
            b2.scols = (int2 *)c->b_scols.p;
            std::vector<BestRec> pb2;
            float ms2 = 0.f;
            rc = run_launch(c, d_seq, tab, b2, bpw, up2, hb2, true, kBatchR, pb2, &ms2, true);
            if (rc != SWB_OK) return rc;
            launches += 2;
            for (size_t k = 0; k < tr.size(); ++k) {
                const swb_batch_item &it = out->items[tr[k]];
                if (!pb2[k].valid || pb2[k].ho - sc->gap_open != it.score || pb2[k].row != it.end_row ||
                    pb2[k].col != it.end_col)
                    return ctx_fail(c, SWB_ECUDA, "batch: store pass disagrees with the scoring pass");
            }
        }
        ph.mark("store pass");
        if (!tr.empty()) {
            const int kS = tb::state_slots();
            // per traced pair: walker state, reversed ops / crosspoints and their capacities
            std::vector<const int64_t *> tS(tr.size()), tX(tr.size());
            std::vector<const char *> tO(tr.size());
            std::vector<int64_t> tOc(tr.size()), tXc(tr.size());
            std::vector<int64_t> st;
            std::vector<char> hops;
            std::vector<int64_t> hxp;
            if (use_graph && first_stores) {
                // the graph walked every pair with a positive score already
                std::vector<int64_t> pos((size_t)npairs, -1);
                for (size_t k = 0; k < order.size(); ++k) pos[(size_t)order[k]] = (int64_t)k;
                for (size_t k = 0; k < tr.size(); ++k) {
                    const size_t q = (size_t)pos[(size_t)tr[k]];
                    tS[k] = gp.states + (size_t)kS * q;
                    tO[k] = gp.ops + gp.ops_off[q];
                    tX[k] = gp.xps + 4 * gp.xp_off[q];
                    tOc[k] = gp.ops_cap[q];
                    tXc[k] = gp.xp_cap[q];
                }
            } else {
                ops_total = xp_total = 0;
                for (size_t k = 0; k < tr.size(); ++k) {
                    ops_total += (int64_t)bpw[k].m + bpw[k].n + 8;
                    xp_total += bpw[k].m / out->items[tr[k]].xpoint_interval + 8;
                }
                if ((e = c->b_ops.ensure((size_t)std::max<int64_t>(1, ops_total))) != cudaSuccess ||
                    (e = c->b_xps.ensure(sizeof(int64_t) * 4 * (size_t)std::max<int64_t>(1, xp_total))) != cudaSuccess ||
                    (e = c->b_state.ensure(sizeof(int64_t) * kS * std::max<size_t>(1, tr.size()))) != cudaSuccess ||
                    (e = c->b_walk.ensure(tb::walk_args_bytes() * std::max<size_t>(1, tr.size()))) != cudaSuccess ||
                    (e = c->b_gdir.ensure(tb::walk_batch_dir_bytes(c->sms, (int64_t)tr.size()))) != cudaSuccess)
                    return ctx_cuda_fail(c, e, "batch traceback buffers");
                std::vector<tb::WalkInputs> win(tr.size());
                st.assign((size_t)kS * tr.size(), 0);
                int64_t oo = 0, xo = 0;
                std::vector<int64_t> ops_off(tr.size()), xp_off(tr.size());
                for (size_t k = 0; k < tr.size(); ++k) {
                    const swb_batch_item &it = out->items[tr[k]];
                    const BatchPair &d = bpw[k];
                    tb::WalkInputs &w = win[k];
                    w.rows = d_seq + d.row_off;
                    w.cols = d_seq + d.col_off;
                    w.m = d.m;
                    w.n = d.n;
                    w.sc = *sc;
                    w.score = it.score;
                    w.srows = (const int2 *)c->b_srows.p + d.sr_off;
                    w.scols = (const int2 *)c->b_scols.p + d.sc_off;
                    w.rr0 = 0;
                    w.cc0 = 0;
                    w.rr1 = d.m;
                    w.cc1 = d.n;
                    w.rtop = nullptr;
                    w.rleft = nullptr;
                    w.xp_interval = it.xpoint_interval;
                    w.ops = (char *)c->b_ops.p + oo;
                    w.ops_cap = (int64_t)d.m + d.n + 8;
                    w.xps = (int64_t *)c->b_xps.p + 4 * xo;
                    w.xp_cap = d.m / it.xpoint_interval + 8;
                    ops_off[k] = oo;
                    xp_off[k] = xo;
                    oo += w.ops_cap;
                    xo += w.xp_cap;
                    int64_t *S = st.data() + (size_t)kS * k;
                    S[tb::slot_r()] = it.end_row;
                    S[tb::slot_c()] = it.end_col;
                }
                std::string err;
                tb::Scratch scr{};
                scr.owner = c;
                scr.get = [](void *owner, void *dst, const void *src, size_t bytes) -> cudaError_t {
                    return ctx_get((swb_ctx *)owner, dst, src, bytes);
                };
                scr.put = [](void *owner, void *dst, const void *src, size_t bytes) -> cudaError_t {
                    return ctx_put((swb_ctx *)owner, dst, src, bytes);
                };
                int rc = tb::walk_batch(c->stream, c->sms, win.data(), (int64_t)win.size(), c->b_walk.p,
                                        (int64_t *)c->b_state.p, c->b_gdir.p, st.data(), scr, err);
                if (rc != SWB_OK) return ctx_fail(c, rc, "%s", err.c_str());
                launches += 1;
                hops.resize((size_t)std::max<int64_t>(1, oo));
                hxp.resize((size_t)std::max<int64_t>(4, 4 * xo));
                if ((e = ctx_get(c, hops.data(), c->b_ops.p, (size_t)oo)) != cudaSuccess ||
                    (e = ctx_get(c, hxp.data(), c->b_xps.p, sizeof(int64_t) * 4 * (size_t)xo)) != cudaSuccess)
                    return ctx_cuda_fail(c, e, "batch traceback copy");
                for (size_t k = 0; k < tr.size(); ++k) {
                    tS[k] = st.data() + (size_t)kS * k;
                    tO[k] = hops.data() + ops_off[k];
                    tX[k] = hxp.data() + 4 * xp_off[k];
                    tOc[k] = win[k].ops_cap;
                    tXc[k] = win[k].xp_cap;
                }
            }
            ph.mark("walker");
            // gather: ops (end -> start on the device) and crosspoints
            int64_t tot_ops = 0, tot_xp = 0;
            for (size_t k = 0; k < tr.size(); ++k) {
                const int64_t *S = tS[k];
                if (S[tb::slot_nops()] > tOc[k] || S[tb::slot_nxp()] > tXc[k])
                    return ctx_fail(c, SWB_ECUDA, "batch traceback output larger than its buffers");
                tot_ops += S[tb::slot_nops()];
                tot_xp += S[tb::slot_nxp()] + 2;
            }
            out->ops = (char *)std::malloc((size_t)tot_ops + 1);
            out->xpoints = (swb_xpoint *)std::malloc(sizeof(swb_xpoint) * (size_t)(tot_xp + 2 * ntrace + 1));
            if (!out->ops || !out->xpoints) return ctx_fail(c, SWB_ENOMEM, "out of host memory");
            int64_t po = 0, px = 0;
            for (size_t k = 0; k < tr.size(); ++k) {
                swb_batch_item &it = out->items[tr[k]];
                const int64_t *S = tS[k];
                const int64_t nops = S[tb::slot_nops()], nxp = S[tb::slot_nxp()];
                it.ops_off = po;
                it.n_ops = nops;
                std::reverse_copy(tO[k], tO[k] + nops, out->ops + po);
                po += nops;
                it.start_row = S[tb::slot_start_r()];
                it.start_col = S[tb::slot_start_c()];
                it.xp_off = px;
                out->xpoints[px++] = swb_xpoint{0, 0, it.start_row, it.start_col};
                for (int64_t q = nxp - 1; q >= 0; --q) {
                    const int64_t *d = tX[k] + 4 * q;
                    out->xpoints[px++] = swb_xpoint{(int32_t)d[3], (int32_t)d[2], d[0], d[1]};
                }
                out->xpoints[px++] = swb_xpoint{0, it.score, it.end_row, it.end_col};
                it.n_xpoints = px - it.xp_off;
            }
            out->ops_bytes = po;
            out->ops[po] = 0;
            out->n_xpoints = px;
        }
        // traced pairs with score 0: no alignment; crosspoints [start = end]
        // (pairs with an empty sequence have none, as in swb_align_pair)
        for (int64_t i : byscore) {
            swb_batch_item &it = out->items[i];
            if (it.score > 0 || info[(size_t)i].n == 0) continue;
            if (!out->xpoints) {
                out->xpoints = (swb_xpoint *)std::malloc(sizeof(swb_xpoint) * (size_t)(ntrace + 1));
                if (!out->xpoints) return ctx_fail(c, SWB_ENOMEM, "out of host memory");
            }
            it.xp_off = out->n_xpoints;
            it.n_xpoints = 1;
            out->xpoints[out->n_xpoints++] = swb_xpoint{0, 0, it.end_row, it.end_col};
        }
        out->stage2_ms = (use_graph && first_stores ? (double)gp.ms2 : 0.0) +
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
    }
    ph.mark("results");
    out->kernel_launches = launches;
    out->total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return SWB_OK;
}

}  // namespace

int batch_align_all_traced(swb_ctx *c, const uint8_t *h_seq, int64_t seq_bytes, const swb_pair_ref *pairs,
                           int64_t npairs, const swb_scoring *sc, uint32_t flags, swb_batch_result *out) {
    int rc = batch_run(c, h_seq, nullptr, seq_bytes, pairs, npairs, sc, flags, 1.0, out, true);
    if (rc != SWB_OK) swb_batch_result_free(out);
    return rc;
}

}  // namespace swb

extern "C" int swb_batch_align(swb_ctx *c, const uint8_t *seq, int64_t seq_bytes, const swb_pair_ref *pairs,
                               int64_t npairs, const swb_scoring *sc, uint32_t flags, double trace_frac,
                               swb_batch_result *out) {
    if (!c || !out || (seq_bytes > 0 && !seq)) return swb::ctx_fail(c, SWB_EINVAL, "swb_batch_align: bad arguments");
    int rc = swb::batch_run(c, seq, nullptr, seq_bytes, pairs, npairs, sc, flags, trace_frac, out, trace_frac >= 1.0);
    if (rc != SWB_OK) swb_batch_result_free(out);
    return rc;
}

extern "C" int swb_batch_align_device(swb_ctx *c, const void *d_seq, int64_t seq_bytes, const swb_pair_ref *pairs,
                                      int64_t npairs, const swb_scoring *sc, uint32_t flags, double trace_frac,
                                      swb_batch_result *out) {
    if (!c || !out || (seq_bytes > 0 && !d_seq))
        return swb::ctx_fail(c, SWB_EINVAL, "swb_batch_align_device: bad arguments");
    int rc = swb::batch_run(c, nullptr, (const uint8_t *)d_seq, seq_bytes, pairs, npairs, sc, flags, trace_frac, out,
                            trace_frac >= 1.0);
    if (rc != SWB_OK) swb_batch_result_free(out);
    return rc;
}

extern "C" void swb_batch_result_free(swb_batch_result *r) {
    if (!r) return;
    std::free(r->items);
    std::free(r->ops);
    std::free(r->xpoints);
    std::memset(r, 0, sizeof *r);
}
