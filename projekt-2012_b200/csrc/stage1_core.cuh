// stage1_core.cuh -- device core of the scoring wavefront, shared by the pair
// kernel (stage1.cu) and the batched kernel (batch.cu).
//
// Follows the recurrence of the reference's shortPhase/longPhase kernels
// (src/FindAlignment.cuh:50-104, twin :187-241) with this library's own layout: a
// warp owns a strip of 32*R rows, lane l owns R consecutive rows and computes
// column k - l at step k; see stage1.cu for the full description.
//
// Every function is templated on the argument type A, which provides the
// fields of Stage1Args that the core reads: the scoring scalars (open, ext, gx,
// mt1, mm1, tab_hi), the error words (err), the sequences or their encodings
// (rows, cols, rcode, ctab), the rectangle (m, n, r_origin, c_origin, top, left,
// corner), the strip handoff buffer (hbuf), the optional stores (srows,
// sr_every, scols, sc_every), the tie geometry (tie) and the running best H of
// the matrix (gbest).  The pair kernel passes Stage1Args itself; the batched
// kernel passes a per-pair view whose unused fields are compile-time nulls.
#pragma once

#include <climits>

#include "swb_internal.h"

namespace swb {
namespace {

constexpr int kCH = 8;         // steps per refill
constexpr int kRing = 32;      // ring entries per warp
constexpr int kStage = 16;     // staged bottom-row entries per warp (flushed every refill)
constexpr int kWarps = 4;      // warps per block
constexpr long long kWaitLimitCycles = 40LL * 1000 * 1000 * 1000;  // default bound of every wait (~20 s)

enum : int32_t { kErrNone = 0, kErrTimeout = 4 };

__device__ __forceinline__ int32_t ld_volatile(const int32_t *p) {
    return *reinterpret_cast<const volatile int32_t *>(p);
}
// LL loads/stores are volatile asm (never removed, merged or reordered with
// each other); they carry no "memory" clobber so the compiler may keep the
// kernel's scalar parameters in registers across them.
__device__ __forceinline__ int4 ld_ll(const int4 *p) {
    int4 v;
    asm volatile("ld.volatile.global.v4.s32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}
__device__ __forceinline__ void st_ll(int4 *p, int32_t ho, int32_t f, int32_t tag) {
    asm volatile("st.volatile.global.v4.s32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(ho), "r"(tag), "r"(f), "r"(tag));
}
// Byte permute with per-nibble sign replication (PTX prmt default mode).
__device__ __forceinline__ int32_t prmt(uint32_t lo, uint32_t hi, uint32_t sel) {
    int32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(lo), "r"(hi), "r"(sel));
    return r;
}

__device__ __forceinline__ uint64_t tie_key(const TieGeom g, int64_t r, int64_t c) {
    if (g.mode == kTieRowMajor) return ((uint64_t)r << 32) | (uint64_t)c;
    // rows and columns are below 2^31: 32-bit arithmetic
    const uint32_t T = (uint32_t)g.T, G = (uint32_t)g.G, C = (uint32_t)g.C;
    const uint32_t r32 = (uint32_t)r, c32 = (uint32_t)c;
    const uint32_t q = r32 >> 2;
    const uint32_t t = q % T;
    const uint32_t s = q / T;
    const uint32_t k = (c32 + t) / C;
    const uint32_t b = G - 1 - (k % G);
    return ((uint64_t)(b * T + t) << 60) | ((uint64_t)(s + k) << 32) | ((uint64_t)(c32 + t - k * C) << 2) |
           (uint64_t)(r32 & 3);
}

__device__ __forceinline__ bool better(int32_t ho, uint64_t key, int32_t bho, uint64_t bkey) {
    return ho > bho || (ho == bho && key < bkey);
}

// A lane's best cell.  Its tie key is computed when first needed: along an
// alignment path almost every new best is strictly better than the lane's
// previous one and alone in its column, so no key is compared (evaluating the
// reference key there, with its integer divisions, at every column the path
// crosses made each strip's slow steps, and through the strip chain the whole
// pass, about 13% slower on the 1 Mbp pair).
struct Best {
    int32_t ho;
    int32_t keyed;   // key holds the tie key of (row, col); else it is computed on demand
    uint64_t key;    // ~0: no cell yet
    int64_t row, col;
};

__device__ __forceinline__ void init_best(Best &b, int32_t open) {
    b.ho = open + 1;  // only H >= 1 is recorded
    b.keyed = 1;
    b.key = ~0ULL;
    b.row = 0;
    b.col = 0;
}

__device__ __forceinline__ void key_best(Best *b, const TieGeom tie, int64_t r_origin, int64_t c_origin) {
    if (!b->keyed) {
        b->key = tie_key(tie, r_origin + b->row, c_origin + b->col);
        b->keyed = 1;
    }
}

// Rows of `mask` hold the column maximum cm at column j: keep the smallest key.
__device__ __forceinline__ int32_t slow_best(uint32_t mask, int32_t cm, const TieGeom tie, int64_t m, int64_t r_origin,
                                          int64_t c_origin, Best *b, int64_t row0, int32_t j, int32_t *gbest,
                                          int32_t open) {
    const int32_t before = b->ho;
    while (mask) {
        const int i = __ffs(mask) - 1;
        mask &= mask - 1;
        const int64_t r = row0 + i;
        if (r >= m) break;
        if (cm > b->ho) {  // strictly better: its key is needed only if a tie comes later
            b->ho = cm;
            b->keyed = 0;
            b->row = r;
            b->col = j;
            continue;
        }
        // cm == b->ho (the candidate test admits nothing below the lane's best)
        key_best(b, tie, r_origin, c_origin);
        const uint64_t key = tie_key(tie, r_origin + r, c_origin + j);
        if (key < b->key) {
            b->key = key;
            b->row = r;
            b->col = j;
        }
    }
    if (b->ho > before) atomicMax(gbest, b->ho - open);
    return b->ho;
}

// The same update with the rows past the end masked first and a single
// strictly-better cell taken without a loop.  The packed batch kernel runs
// about 5% faster with this form; the single-pair kernels with slow_best
// (code layout of the two differs; both give the same cell).
__device__ __forceinline__ int32_t slow_best_single(uint32_t mask, int32_t cm, const TieGeom tie, int64_t m,
                                                 int64_t r_origin, int64_t c_origin, Best *b, int64_t row0,
                                                 int32_t j, int32_t *gbest, int32_t open) {
    const int32_t before = b->ho;
    if (row0 + 32 > m) mask &= (m - row0 > 0) ? (uint32_t)((1ULL << (m - row0)) - 1ULL) : 0u;
    if (mask == 0) return b->ho;
    if (cm > b->ho && (mask & (mask - 1)) == 0) {
        b->ho = cm;
        b->keyed = 0;
        b->row = row0 + __ffs(mask) - 1;
        b->col = j;
    } else {
        key_best(b, tie, r_origin, c_origin);
        while (mask) {
            const int i = __ffs(mask) - 1;
            mask &= mask - 1;
            const int64_t r = row0 + i;
            const uint64_t key = tie_key(tie, r_origin + r, c_origin + j);
            if (better(cm, key, b->ho, b->key)) {
                b->ho = cm;
                b->key = key;
                b->row = r;
                b->col = j;
            }
        }
    }
    if (b->ho > before) atomicMax(gbest, b->ho - open);
    return b->ho;
}

template <int R>
struct Lane {
    uint32_t ra[R];  // TAB: prmt selector of the row code; CMP: row byte (256 past the end)
    int32_t HO[R];   // H + open of the previous column
    int32_t E[R];    // E of the previous column
    int32_t inHO, inF;       // from the lane above: HO of its last row, F of my row 0
    uint32_t inB;            // column value: TAB table word / CMP byte
    int32_t hodPrev;         // HO of the row above my row 0 at the previous column
    int32_t hodInit;         // HO of the row above my row 0 left of column 0
    int32_t bho;             // this lane's best HO (copy of best.ho)
    int32_t thr;             // candidate threshold: max(bho, device-wide best H + open)
};

struct StripCtx {
    int64_t row0;     // first row of this lane
    int32_t strip;    // strip index (also the tag it writes)
    int32_t n;
    bool sr;          // this strip's bottom row is a special row
    bool below;       // a strip below this one reads its bottom row from hbuf
    bool last_row;    // this strip's bottom row is the rectangle's last row, kept in a.bottom
    int64_t sr_off;   // srows offset of that row
};

// One anti-diagonal step.  PRED: some lanes of the warp are outside [0, n).
// SC: this step may be a special-column step of some lane.  Lane 31 stages the
// strip's bottom row {H + open, F below, F, -} for its column in shared memory;
// the refill writes the staged columns out (hand-off buffer, special row), so
// the step itself issues no global store.
//
// Phase 1 computes, for every row of the lane, E and t = max(H_diag + s, E, 0)
// (independent of the vertical chain); phase 2 runs the F chain and writes HO.
// Every register of the lane arrays is read before it is overwritten, so no
// copies are needed.  The column maximum is taken over t: a cell whose H comes
// from F is strictly below the cell above it, so it can never hold the best
// score, and a best cell always has H = t.
template <int R, bool TAB, bool PRED, bool SC, class A>
__device__ __forceinline__ void step(Lane<R> &L, const A &a, Best *b, const int4 *ring, int4 *stage, int lane,
                                     const StripCtx &sc, int32_t k) {
    const int32_t j = k - lane;
    const bool act = !PRED || (j >= 0 && j < sc.n);
    const uint32_t cb = L.inB;
    int32_t to[R];
    int32_t hod = (PRED && j == 0) ? L.hodInit : L.hodPrev;
#pragma unroll
    for (int i = 0; i < R; ++i) {
        int32_t s1;
        if (TAB) s1 = prmt(cb, a.tab_hi, L.ra[i]);
        else s1 = (L.ra[i] == cb) ? a.mt1 : a.mm1;
        const int32_t e = __viaddmax_s32(L.E[i], a.ext, L.HO[i]);
        to[i] = __viaddmax_s32_relu(hod, s1, e) + a.open;
        hod = L.HO[i];
        if (act) L.E[i] = e;
    }
    // column maximum of t as a shallow tree (branch input ready early)
    int32_t cm;
    {
        int32_t l1[(R + 2) / 3];
#pragma unroll
        for (int q = 0; q < (R + 2) / 3; ++q) {
            const int i = 3 * q;
            l1[q] = (i + 2 < R) ? __vimax3_s32(to[i], to[i + 1], to[i + 2]) : (i + 1 < R ? max(to[i], to[i + 1]) : to[i]);
        }
        constexpr int N1 = (R + 2) / 3;
        int32_t l2[(N1 + 2) / 3];
#pragma unroll
        for (int q = 0; q < (N1 + 2) / 3; ++q) {
            const int i = 3 * q;
            l2[q] = (i + 2 < N1) ? __vimax3_s32(l1[i], l1[i + 1], l1[i + 2]) : (i + 1 < N1 ? max(l1[i], l1[i + 1]) : l1[i]);
        }
        constexpr int N2 = (N1 + 2) / 3;
        cm = l2[0];
#pragma unroll
        for (int q = 1; q < N2; ++q) cm = max(cm, l2[q]);
    }
    int32_t f = L.inF;
    int32_t flast = 0;
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int32_t ho = __viaddmax_s32(f, a.open, to[i]);
        flast = f;
        f = __viaddmax_s32(f, a.gx, to[i]);
        if (act) L.HO[i] = ho;
    }

    // outputs toward the lane below; lane 31 hands its slot to lane 0
    const int4 rv = ring[(k + 1) & (kRing - 1)];
    const bool last = (lane == 31);
    if (last && act) stage[j & (kStage - 1)] = make_int4(L.HO[R - 1], f, flast, 0);
    const int32_t oHO = last ? rv.x : L.HO[R - 1];
    const int32_t oF = last ? rv.y : f;
    const uint32_t oB = last ? (uint32_t)rv.z : cb;
    L.hodPrev = L.inHO;
    const int src = (lane + 31) & 31;
    L.inHO = __shfl_sync(0xffffffffu, oHO, src);
    L.inF = __shfl_sync(0xffffffffu, oF, src);
    L.inB = __shfl_sync(0xffffffffu, oB, src);

    if (act && cm >= L.thr) {
        // rows holding cm in H: every row whose H = t = cm is among them (a row
        // with HO == cm but t < cm takes H from F and can never be the best)
        uint32_t mask = 0;
#pragma unroll
        for (int i = 0; i < R; ++i) mask |= (L.HO[i] == cm ? 1u : 0u) << i;
        L.bho = slow_best(mask, cm, a.tie, a.m, a.r_origin, a.c_origin, b, sc.row0, j, a.gbest, a.open);
        L.thr = max(L.thr, L.bho);
    }
    if (SC && act && ((j + 1) & (a.sc_every - 1)) == 0) {
        // two rows per 16-byte store when the lane's rows are whole and aligned
        // (measured on the 1 Mbp pair: 693 -> 667 ms for the store pass; staging the
        // column in shared memory for 512-byte coalesced stores measured 672 ms,
        // streaming stores 671 ms)
        int2 *dst = a.scols + (int64_t)((j + 1) / a.sc_every - 1) * a.m + sc.row0;
        if (sc.row0 + R <= a.m && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
#pragma unroll
            for (int i = 0; i < R; i += 2)
                reinterpret_cast<int4 *>(dst)[i / 2] =
                    make_int4(L.HO[i] - a.open, L.E[i], L.HO[i + 1] - a.open, L.E[i + 1]);
        } else {
#pragma unroll
            for (int i = 0; i < R; ++i)
                if (sc.row0 + i < a.m) dst[i] = make_int2(L.HO[i] - a.open, L.E[i]);
        }
    }
}

// Column value of column c: the table word (TAB) or the byte (CMP).
template <bool TAB, class A>
__device__ __forceinline__ uint32_t col_value(const A &a, int32_t c) {
    if (TAB) return a.ctab[c];
    return (uint32_t)a.cols[c];
}

// Prefetched inputs of one ring entry (held in registers for one refill).
struct Pre {
    int4 h;        // hbuf entry (strip > 0) or top boundary values (strip 0)
    uint32_t cv;   // column value
};

template <bool TAB, class A>
__device__ __forceinline__ void prefetch(const A &a, int32_t strip, int32_t c, Pre &p) {
    p.cv = col_value<TAB>(a, c);
    if (strip > 0) {
        p.h = ld_ll(a.hbuf + c);
    } else if (a.top) {
        const int2 t = a.top[c];
        p.h.x = t.x + a.open;
        p.h.y = 0;
        p.h.z = max(t.y + a.ext, t.x + a.open);
        p.h.w = 0;
    } else {
        p.h.x = a.open;  // H = 0 above the first row
        p.h.y = 0;
        p.h.z = a.gx;    // F of row 0 = max(0 + ext, 0 + open)
        p.h.w = 0;
    }
}

// Stores the prefetched entry of column c into the ring (re-polling until the
// strip above has written it).  Returns false on timeout/abort.
template <class A>
__device__ __forceinline__ bool commit(const A &a, int4 *ring, int32_t strip, int32_t c, Pre &p) {
    if (strip > 0 && (p.h.y != strip - 1 || p.h.w != strip - 1)) {
        const long long t0 = clock64();
        const long long limit = a.wait_limit > 0 ? a.wait_limit : kWaitLimitCycles;
        for (;;) {
            __nanosleep(32);
            p.h = ld_ll(a.hbuf + c);
            if (p.h.y == strip - 1 && p.h.w == strip - 1) break;
            if (ld_volatile(&a.err[1]) != 0 || clock64() - t0 > limit) return false;
        }
    }
    ring[c & (kRing - 1)] = make_int4(p.h.x, p.h.z, (int32_t)p.cv, 0);
    return true;
}

// Refill at step k (k % kCH == 0): lanes 0..kCH-1 commit columns [k+kCH, k+2kCH)
// (prefetched one refill ago) and prefetch columns [k+2kCH, k+3kCH).
// Writes out the bottom-row columns lane 31 staged in the 8 steps before step k:
// columns [k - kCH - 31, k - 31) (lanes 0..kCH-1, one column each): the
// hand-off entry for the strip below and, for a special row, (H, F).
template <class A>
__device__ __forceinline__ void flush(const A &a, const int4 *stage, int lane, const StripCtx &sc, int32_t n,
                                      int32_t k) {
    __syncwarp();
    if (lane < kCH && (sc.below || sc.sr || sc.last_row)) {
        const int32_t c = k - kCH - 31 + lane;
        if (c >= 0 && c < n) {
            const int4 v = stage[c & (kStage - 1)];
            if (sc.below) st_ll(a.hbuf + c, v.x, v.y, sc.strip);
            if (sc.sr) a.srows[sc.sr_off + c] = make_int2(v.x - a.open, v.z);
            if (sc.last_row) a.bottom[c] = make_int2(v.x - a.open, v.z);
        }
    }
}

template <bool TAB, class A>
__device__ __forceinline__ bool refill(const A &a, int4 *ring, const int4 *stage, int lane, const StripCtx &sc,
                                       int32_t n, int32_t k, Pre &pre, int32_t &thr, int32_t bho, int32_t &gpre) {
    const int32_t strip = sc.strip;
    flush(a, stage, lane, sc, n, k);
    // cells below the best H found anywhere so far can never win: raise the
    // candidate threshold to it (ties at that value are still examined); the
    // value was loaded one refill ago
    thr = max(bho, max(thr, gpre + a.open));
    gpre = ld_volatile(a.gbest);
    bool ok = true;
    if (lane < kCH) {
        const int32_t c = k + kCH + lane;
        if (c < n) ok = commit(a, ring, strip, c, pre);
        const int32_t cn = c + kCH;
        if (cn < n) prefetch<TAB>(a, strip, cn, pre);
    }
    const bool all_ok = __all_sync(0xffffffffu, ok);
    __syncwarp();
    return all_ok;
}

// STORES: the launch may write special rows or columns (a.srows or a.scols set).
// UNROLL: unroll the plain 8-step chunks.  Kernels are instantiated per mode so
// that each holds only the step bodies it runs (the step loop's speed depends on
// what else is compiled into it).
template <int R, bool TAB, bool STORES, bool UNROLL, class A>
__device__ bool run_strip(const A &a, int4 *ring, int4 *stage, int lane, int32_t s, Best *b, int32_t &bho) {
    Lane<R> L;
    StripCtx sc;
    const int64_t H = 32LL * R;
    sc.row0 = (int64_t)s * H + (int64_t)lane * R;
    sc.strip = s;
    sc.n = (int32_t)a.n;
    sc.below = (int64_t)(s + 1) * H < a.m && !(a.withhold && s == 0);
    // the block outputs (swb_score_block_device) come from score-only launches
    sc.last_row = !STORES && a.bottom != nullptr && (int64_t)(s + 1) * H == a.m;
    sc.sr = a.srows != nullptr && ((int64_t)(s + 1) % a.sr_every) == 0 && (int64_t)(s + 1) * H <= a.m;
    sc.sr_off = sc.sr ? ((int64_t)(s + 1) / a.sr_every - 1) * a.n : 0;
    L.bho = bho;
    int32_t gpre = ld_volatile(a.gbest);
    L.thr = max(bho, gpre + a.open);
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int64_t r = sc.row0 + i;
        const bool in = r < a.m;
        if (TAB) {
            const uint32_t q = in ? (uint32_t)a.rcode[r] : 7u;  // code 7 never matches
            const uint32_t qs = q | 8u;
            L.ra[i] = q | (qs << 4) | (qs << 8) | (qs << 12);
        } else {
            L.ra[i] = in ? (uint32_t)a.rows[r] : 256u;
        }
        if (a.left && in) {
            const int2 lv = a.left[r];
            L.HO[i] = lv.x + a.open;
            L.E[i] = lv.y;
        } else {
            L.HO[i] = a.open;  // H = 0 left of column 0
            L.E[i] = 0;        // E = 0 left of column 0 (the reference's zeroed buffer)
        }
    }
    if (sc.row0 == 0) L.hodInit = a.corner + a.open;
    else if (a.left && sc.row0 - 1 < a.m) L.hodInit = a.left[sc.row0 - 1].x + a.open;
    else L.hodInit = a.open;

    const int32_t n = sc.n;
    // prologue: ring entries for columns [0, 2kCH); prefetch [2kCH, 3kCH)
    Pre pre;
    bool ok = true;
    if (lane < kCH) {
        for (int32_t c = lane; c < 2 * kCH && ok; c += kCH) {
            if (c < n) {
                prefetch<TAB>(a, s, c, pre);
                ok = commit(a, ring, s, c, pre);
            }
        }
        if (2 * kCH + lane < n) prefetch<TAB>(a, s, 2 * kCH + lane, pre);
    }
    if (!__all_sync(0xffffffffu, ok)) return false;
    __syncwarp();
    if (a.trace && lane == 0) {  // prologue done: the strip above has delivered columns [0, 2kCH)
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        a.trace[3 * s] = (int64_t)t;
    }
    {
        const int4 v = ring[0];
        L.inHO = v.x;
        L.inF = v.y;
        L.inB = (uint32_t)v.z;
        L.hodPrev = L.hodInit;
    }

    // Steps: [0, 32) ramp-up (predicated), [32, kB) steady, [kB, n + 31) ramp-down.
    // Refills at every multiple of kCH except 0.  In the steady part, only the
    // 32 steps after a multiple of sc_every hold special-column stores.
    const int32_t kEnd = n + 31;
    const int32_t kA = min(32, kEnd);
    int32_t kB = kA;
    if (n > 32) kB = 32 + ((n - 32) / kCH) * kCH;
    int32_t k = 0;
    for (; k < kA; ++k) {
        if (k > 0 && (k % kCH) == 0 && !refill<TAB>(a, ring, stage, lane, sc, n, k, pre, L.thr, L.bho, gpre)) return false;
        if constexpr (!STORES) step<R, TAB, true, false>(L, a, b, ring, stage, lane, sc, k);
        else if (a.scols) step<R, TAB, true, true>(L, a, b, ring, stage, lane, sc, k);
        else step<R, TAB, true, false>(L, a, b, ring, stage, lane, sc, k);
    }
    while (k < kB) {
        if (!refill<TAB>(a, ring, stage, lane, sc, n, k, pre, L.thr, L.bho, gpre)) return false;
        // lane l stores special column j = q*sc_every - 1 at step j + l: a chunk of
        // steps [k, k+kCH) needs the check when some (t + 1) mod sc_every < 32
        const bool sc_window = a.scols != nullptr && ((k + kCH) & (a.sc_every - 1)) < 32 + kCH;
        // The pair kernel's score-only launches unroll the chunk fully, launches
        // with stores by 4 outside the special-column windows, the batched
        // score-only kernel not at all (measured on the 1 Mbp pair: the full
        // unroll saves 5-8% of the score-only time but costs the store-mode
        // kernel 20-27% and the batched kernel about 50%; unrolled by 4 the
        // store-mode kernel is 5.4% faster than rolled, 563.8 vs 595.8 ms, and
        // 1.9% on the 10 Mbp pair; by 2, 568.4 ms).
        if (STORES && sc_window) {
            for (int u = 0; u < kCH; ++u) step<R, TAB, false, true>(L, a, b, ring, stage, lane, sc, k + u);
        } else if constexpr (UNROLL) {
#pragma unroll
            for (int u = 0; u < kCH; ++u) step<R, TAB, false, false>(L, a, b, ring, stage, lane, sc, k + u);
        } else if constexpr (STORES) {
#pragma unroll 4
            for (int u = 0; u < kCH; ++u) step<R, TAB, false, false>(L, a, b, ring, stage, lane, sc, k + u);
        } else {
            for (int u = 0; u < kCH; ++u) step<R, TAB, false, false>(L, a, b, ring, stage, lane, sc, k + u);
        }
        k += kCH;
    }
    for (; k < kEnd; ++k) {
        if ((k % kCH) == 0 && !refill<TAB>(a, ring, stage, lane, sc, n, k, pre, L.thr, L.bho, gpre)) return false;
        if constexpr (!STORES) step<R, TAB, true, false>(L, a, b, ring, stage, lane, sc, k);
        else if (a.scols) step<R, TAB, true, true>(L, a, b, ring, stage, lane, sc, k);
        else step<R, TAB, true, false>(L, a, b, ring, stage, lane, sc, k);
    }
    // the columns staged since the last refill
    flush(a, stage, lane, sc, n, ((kEnd + kCH - 1) / kCH) * kCH);
    __syncwarp();
    if (!STORES && a.right != nullptr) {
        // after its last column a lane's registers hold H + open and E of column n - 1
#pragma unroll
        for (int i = 0; i < R; ++i)
            if (sc.row0 + i < a.m) a.right[sc.row0 + i] = make_int2(L.HO[i] - a.open, L.E[i]);
    }
    bho = L.bho;
    return true;
}

}  // namespace
}  // namespace swb
