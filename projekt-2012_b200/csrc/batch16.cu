// batch16.cu -- the scoring pass of a batch with two pairs per warp in packed
// 16-bit lanes (int16x2 DPX).
//
// No counterpart in the reference, whose recurrence is int32 only
// (src/FindAlignment.cuh:54-56).  Every 32-bit register of a lane holds the same
// row of two pairs: pair a in the low half, pair b in the high half, so each DPX
// instruction (__viaddmax_s16x2 and friends, one instruction at the rate of the
// int32 ones) updates two cells.  The recurrence is the one of stage1_core.cuh
// on H + open, per half:
//     E  = max(E_left + ext, HO_left)           __viaddmax_s16x2
//     t  = max(HO_diag + (s - open), E, 0)      __viaddmax_s16x2_relu
//     HO = max(F + open, t + open), F' = max(F + max(ext, open), t + open)
// One PRMT per row yields both halves' substitution scores: the selector takes
// byte q_a of pair a's column word with its sign replicated into the next byte,
// and byte q_b of pair b's column word likewise (table words as in TAB mode).
//
// Exactness.  Every value stays at or above gap_open (t >= 0, E >= HO_left,
// F' >= t + open), so the low end never wraps.  The high end is bounded by the
// host: a pair is packed only when match * (shorter length) + 256 <= 32,767, so
// no cell can exceed the half's range.  The kernel checks it anyway: a column
// maximum at or above `sat_lim` in a half sets that pair's saturation flag, and
// the host scores flagged pairs again in int32 (a cell can grow by at most
// `match` per diagonal step, so the first cell past sat_lim is seen before any
// value wraps).  Results are identical to the int32 path; the tests force
// saturation on a pair that cannot fit and check the int32 answer.
//
// Pairs a and b of one packed unit have the same strip count (the host pairs
// pairs of similar size); the packed rectangle is max(m) x max(n).  Rows past a
// half's pair get code 0 and columns past it the all-mismatch word: those cells
// only feed cells further down or right, never a cell of the pair, and the slow
// path ignores them.  The strips of a packed pair are chained through one
// hand-off buffer of packed entries {HO, tag, F, tag} exactly as in
// stage1_core.cuh, with the same bounded waits.
#include <algorithm>

#include "batch.h"
#include "stage1_core.cuh"

namespace swb {
namespace {

template <int R>
struct Lane16 {
    uint32_t ra[R];      // prmt selectors (both halves' row codes)
    uint32_t HO[R];      // packed H + open of the previous column
    uint32_t E[R];       // packed E of the previous column
    uint32_t inHO, inF;  // from the lane above
    uint32_t inA, inB;   // column words of pair a and pair b
    uint32_t hodPrev;
    uint32_t thr;        // packed candidate thresholds
};

__device__ __forceinline__ int32_t half(uint32_t v, int h) { return (int32_t)(int16_t)(uint16_t)(v >> (16 * h)); }
__device__ __forceinline__ uint32_t pack2(int32_t lo, int32_t hi) {
    return ((uint32_t)(uint16_t)(int16_t)lo) | ((uint32_t)(uint16_t)(int16_t)hi << 16);
}

struct Pre16 {
    int4 h;
    uint32_t wa, wb;
};

struct Strip16 {
    int64_t row0;
    int32_t strip;
    bool below;
};

__device__ __forceinline__ void prefetch16(const Batch16Args &g, const PackedPair &d, int32_t s, int32_t c, Pre16 &p) {
    p.wa = c < d.n[0] ? g.ctab[d.col_off[0] + c] : g.mm4;
    p.wb = c < d.n[1] ? g.ctab[d.col_off[1] + c] : g.mm4;
    if (s > 0) {
        p.h = ld_ll(g.hbuf + d.hbuf_off + c);
    } else {
        p.h.x = (int32_t)g.open2;  // H = 0 above the first row
        p.h.y = 0;
        p.h.z = (int32_t)g.gx2;    // F of row 0
        p.h.w = 0;
    }
}

__device__ __forceinline__ bool commit16(const Batch16Args &g, const PackedPair &d, int4 *ring, int32_t s, int32_t c,
                                         Pre16 &p) {
    if (s > 0 && (p.h.y != s - 1 || p.h.w != s - 1)) {
        const long long t0 = clock64();
        const long long limit = g.wait_limit > 0 ? g.wait_limit : kWaitLimitCycles;
        for (;;) {
            __nanosleep(32);
            p.h = ld_ll(g.hbuf + d.hbuf_off + c);
            if (p.h.y == s - 1 && p.h.w == s - 1) break;
            if (ld_volatile(&g.ctl[2]) != 0 || clock64() - t0 > limit) return false;
        }
    }
    ring[c & (kRing - 1)] = make_int4(p.h.x, p.h.z, (int32_t)p.wa, (int32_t)p.wb);
    return true;
}

__device__ __forceinline__ void flush16(const Batch16Args &g, const PackedPair &d, const int4 *stage, int lane,
                                        const Strip16 &sc, int32_t n, int32_t k) {
    __syncwarp();
    if (lane < kCH && sc.below) {
        const int32_t c = k - kCH - 31 + lane;
        if (c >= 0 && c < n) {
            const int4 v = stage[c & (kStage - 1)];
            st_ll(g.hbuf + d.hbuf_off + c, v.x, v.y, sc.strip);
        }
    }
}

// Half h of the column maximum reached the threshold at column j: record the
// rows holding it (lazy tie keys, as slow_best_single), flag saturation.
template <int R>
__device__ __forceinline__ void slow16(Lane16<R> &L, const Batch16Args &g, const PackedPair &d, Best *b, int h,
                                       uint32_t cm, int64_t row0, int32_t j) {
    if (j >= d.n[h]) return;  // a column past this half's pair
    const int32_t c = half(cm, h);
    if (c >= g.sat_lim) atomicExch(&g.sat[d.slot[h]], 1);
    uint32_t mask = 0;
#pragma unroll
    for (int i = 0; i < R; ++i) mask |= (half(L.HO[i], h) == c ? 1u : 0u) << i;
    const int32_t bho = slow_best_single(mask, c, d.tie[h], d.m[h], 0, 0, b, row0, j, g.gbest + d.slot[h], g.open);
    const int32_t t = half(L.thr, h);
    const int32_t nt = max(t, bho);
    L.thr = h == 0 ? ((L.thr & 0xFFFF0000u) | (uint32_t)(uint16_t)(int16_t)nt)
                   : ((L.thr & 0x0000FFFFu) | ((uint32_t)(uint16_t)(int16_t)nt << 16));
}

template <int R, bool PRED>
__device__ __forceinline__ void step16(Lane16<R> &L, const Batch16Args &g, const PackedPair &d, Best *ba, Best *bb,
                                       const int4 *ring, int4 *stage, int lane, const Strip16 &sc, int32_t k) {
    const int32_t j = k - lane;
    const bool act = !PRED || (j >= 0 && j < d.N);
    const uint32_t wa = L.inA, wb = L.inB;
    uint32_t to[R];
    uint32_t hod = (PRED && j == 0) ? g.open2 : L.hodPrev;
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const uint32_t s1 = (uint32_t)prmt(wa, wb, L.ra[i]);
        const uint32_t e = __viaddmax_s16x2(L.E[i], g.ext2, L.HO[i]);
        to[i] = __vadd2(__viaddmax_s16x2_relu(hod, s1, e), g.open2);
        hod = L.HO[i];
        if (act) L.E[i] = e;
    }
    uint32_t cm;
    {
        uint32_t l1[(R + 2) / 3];
#pragma unroll
        for (int q = 0; q < (R + 2) / 3; ++q) {
            const int i = 3 * q;
            l1[q] = (i + 2 < R) ? __vimax3_s16x2(to[i], to[i + 1], to[i + 2])
                                : (i + 1 < R ? __vmaxs2(to[i], to[i + 1]) : to[i]);
        }
        constexpr int N1 = (R + 2) / 3;
        cm = l1[0];
#pragma unroll
        for (int q = 1; q < N1; ++q) cm = __vmaxs2(cm, l1[q]);
    }
    uint32_t f = L.inF;
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const uint32_t ho = __viaddmax_s16x2(f, g.open2, to[i]);
        f = __viaddmax_s16x2(f, g.gx2, to[i]);
        if (act) L.HO[i] = ho;
    }
    const int4 rv = ring[(k + 1) & (kRing - 1)];
    const bool last = (lane == 31);
    if (last && act) stage[j & (kStage - 1)] = make_int4((int32_t)L.HO[R - 1], (int32_t)f, 0, 0);
    const uint32_t oHO = last ? (uint32_t)rv.x : L.HO[R - 1];
    const uint32_t oF = last ? (uint32_t)rv.y : f;
    const uint32_t oA = last ? (uint32_t)rv.z : wa;
    const uint32_t oB = last ? (uint32_t)rv.w : wb;
    L.hodPrev = L.inHO;
    const int src = (lane + 31) & 31;
    L.inHO = __shfl_sync(0xffffffffu, oHO, src);
    L.inF = __shfl_sync(0xffffffffu, oF, src);
    L.inA = __shfl_sync(0xffffffffu, oA, src);
    L.inB = __shfl_sync(0xffffffffu, oB, src);
    const uint32_t hit = __vcmpges2(cm, L.thr);
    if (act && hit) {
        if (hit & 0xFFFFu) slow16<R>(L, g, d, ba, 0, cm, sc.row0, j);
        if (hit >> 16) slow16<R>(L, g, d, bb, 1, cm, sc.row0, j);
    }
}

template <int R>
__device__ __forceinline__ bool refill16(Lane16<R> &L, const Batch16Args &g, const PackedPair &d, int4 *ring,
                                         const int4 *stage, int lane, const Strip16 &sc, int32_t k, Pre16 &pre,
                                         uint32_t &gpre) {
    flush16(g, d, stage, lane, sc, d.N, k);
    // the best H of each pair found anywhere so far (loaded one refill ago)
    L.thr = __vmaxs2(L.thr, __vadd2(gpre, g.open2));
    gpre = pack2(ld_volatile(g.gbest + d.slot[0]), ld_volatile(g.gbest + d.slot[1]));
    bool ok = true;
    if (lane < kCH) {
        const int32_t c = k + kCH + lane;
        if (c < d.N) ok = commit16(g, d, ring, sc.strip, c, pre);
        const int32_t cn = c + kCH;
        if (cn < d.N) prefetch16(g, d, sc.strip, cn, pre);
    }
    const bool all_ok = __all_sync(0xffffffffu, ok);
    __syncwarp();
    return all_ok;
}

template <int R>
__device__ bool run_strip16(const Batch16Args &g, const PackedPair &d, int4 *ring, int4 *stage, int lane, int32_t s,
                            Best *ba, Best *bb) {
    Lane16<R> L;
    Strip16 sc;
    const int64_t H = 32LL * R;
    sc.row0 = (int64_t)s * H + (int64_t)lane * R;
    sc.strip = s;
    sc.below = (int64_t)(s + 1) * H < d.M;
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int64_t r = sc.row0 + i;
        const uint32_t qa = r < d.m[0] ? (uint32_t)g.rcode[d.row_off[0] + r] : 0u;
        const uint32_t qb = r < d.m[1] ? (uint32_t)g.rcode[d.row_off[1] + r] : 0u;
        L.ra[i] = qa | ((qa | 8u) << 4) | ((qb + 4u) << 8) | (((qb + 4u) | 8u) << 12);
        L.HO[i] = g.open2;  // H = 0 left of column 0
        L.E[i] = 0u;        // E = 0 left of column 0
    }
    L.thr = pack2(ba->ho, bb->ho);
    uint32_t gpre = pack2(ld_volatile(g.gbest + d.slot[0]), ld_volatile(g.gbest + d.slot[1]));
    L.thr = __vmaxs2(L.thr, __vadd2(gpre, g.open2));
    const int32_t n = d.N;
    Pre16 pre;
    bool ok = true;
    if (lane < kCH) {
        for (int32_t c = lane; c < 2 * kCH && ok; c += kCH) {
            if (c < n) {
                prefetch16(g, d, s, c, pre);
                ok = commit16(g, d, ring, s, c, pre);
            }
        }
        if (2 * kCH + lane < n) prefetch16(g, d, s, 2 * kCH + lane, pre);
    }
    if (!__all_sync(0xffffffffu, ok)) return false;
    __syncwarp();
    {
        const int4 v = ring[0];
        L.inHO = (uint32_t)v.x;
        L.inF = (uint32_t)v.y;
        L.inA = (uint32_t)v.z;
        L.inB = (uint32_t)v.w;
        L.hodPrev = g.open2;
    }
    const int32_t kEnd = n + 31;
    const int32_t kA = min(32, kEnd);
    int32_t kB = kA;
    if (n > 32) kB = 32 + ((n - 32) / kCH) * kCH;
    int32_t k = 0;
    for (; k < kA; ++k) {
        if (k > 0 && (k % kCH) == 0 && !refill16<R>(L, g, d, ring, stage, lane, sc, k, pre, gpre)) return false;
        step16<R, true>(L, g, d, ba, bb, ring, stage, lane, sc, k);
    }
    while (k < kB) {
        if (!refill16<R>(L, g, d, ring, stage, lane, sc, k, pre, gpre)) return false;
        for (int u = 0; u < kCH; ++u) step16<R, false>(L, g, d, ba, bb, ring, stage, lane, sc, k + u);
        k += kCH;
    }
    for (; k < kEnd; ++k) {
        if ((k % kCH) == 0 && !refill16<R>(L, g, d, ring, stage, lane, sc, k, pre, gpre)) return false;
        step16<R, true>(L, g, d, ba, bb, ring, stage, lane, sc, k);
    }
    flush16(g, d, stage, lane, sc, n, ((kEnd + kCH - 1) / kCH) * kCH);
    __syncwarp();
    return true;
}

__device__ __forceinline__ void warp_best(Best &b) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const int32_t oho = __shfl_xor_sync(0xffffffffu, b.ho, off);
        const uint64_t okey = __shfl_xor_sync(0xffffffffu, b.key, off);
        const int64_t orow = __shfl_xor_sync(0xffffffffu, b.row, off);
        const int64_t ocol = __shfl_xor_sync(0xffffffffu, b.col, off);
        if (better(oho, okey, b.ho, b.key)) {
            b.ho = oho;
            b.key = okey;
            b.row = orow;
            b.col = ocol;
        }
    }
}

template <int R>
__global__ void __launch_bounds__(kWarps * 32, 4) batch16_kernel(Batch16Args g) {
    __shared__ int4 ring_all[kWarps][kRing + kStage];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    int4 *ring = ring_all[wib];
    int4 *stage = ring + kRing;
    for (;;) {
        __syncwarp();
        int32_t u = 0;
        if (lane == 0) u = atomicAdd(&g.ctl[0], 1);
        u = __shfl_sync(0xffffffffu, u, 0);
        if (u >= g.nunits || ld_volatile(&g.ctl[2]) != 0) break;
        const int2 it = g.items[u];
        // a whole pair: every strip in turn (the strip above is always complete,
        // so no wait ends up spinning); else the item's one strip.  The pair's
        // descriptor is read again for every strip rather than kept live across
        // them (fewer spilled registers: 1% faster on the 100,000-pair batch).
        const int32_t s0 = it.y, s1 = g.pairs[it.x].whole ? g.pairs[it.x].nstrips : s0 + 1;
        bool ok = true;
        for (int32_t s = s0; s < s1 && ok; ++s) {
            const PackedPair d = g.pairs[it.x];
            Best ba, bb;
            init_best(ba, g.open);
            init_best(bb, g.open);
            if (!run_strip16<R>(g, d, ring, stage, lane, s, &ba, &bb)) {
                if (lane == 0) {
                    atomicCAS(&g.ctl[1], kErrNone, kErrTimeout);
                    atomicExch(&g.ctl[2], 1);
                }
                ok = false;
                break;
            }
            key_best(&ba, d.tie[0], 0, 0);
            key_best(&bb, d.tie[1], 0, 0);
            warp_best(ba);
            warp_best(bb);
            if (lane == 0) {
                const int64_t ub = 2 * ((int64_t)d.unit0 + s);
                BestRec r;
                r.ho = ba.ho;
                r.valid = (ba.key != ~0ULL) ? 1 : 0;
                r.key = ba.key;
                r.row = ba.row;
                r.col = ba.col;
                g.ubest[ub] = r;
                r.ho = bb.ho;
                r.valid = (bb.key != ~0ULL) ? 1 : 0;
                r.key = bb.key;
                r.row = bb.row;
                r.col = bb.col;
                g.ubest[ub + 1] = r;
            }
            __syncwarp();
        }
        if (!ok) break;
    }
}

__device__ __forceinline__ void merge16(BestRec &b, const BestRec &r) {
    if (r.valid && (!b.valid || better(r.ho, r.key, b.ho, b.key))) b = r;
}

// A warp per packed pair: each half's unit records into its pair's slot.
__global__ void batch16_reduce_kernel(const PackedPair *pairs, int64_t npairs, const BestRec *ubest, BestRec *pbest) {
    const int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (p >= npairs) return;
    const int lane = threadIdx.x & 31;
    const PackedPair d = pairs[p];
    for (int h = 0; h < 2; ++h) {
        if (d.m[h] == 0) continue;
        BestRec b;
        b.ho = INT_MIN;
        b.valid = 0;
        b.key = ~0ULL;
        b.row = 0;
        b.col = 0;
        for (int32_t u = d.unit0 + lane; u < d.unit0 + d.nstrips; u += 32) merge16(b, ubest[2 * (int64_t)u + h]);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            BestRec o;
            o.ho = __shfl_xor_sync(0xffffffffu, b.ho, off);
            o.valid = __shfl_xor_sync(0xffffffffu, b.valid, off);
            o.key = __shfl_xor_sync(0xffffffffu, b.key, off);
            o.row = __shfl_xor_sync(0xffffffffu, b.row, off);
            o.col = __shfl_xor_sync(0xffffffffu, b.col, off);
            merge16(b, o);
        }
        if (lane == 0) pbest[d.slot[h]] = b;
    }
}

template <int R>
int max_blocks16() {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, batch16_kernel<R>, kWarps * 32, 0) != cudaSuccess) return 0;
    return nb;
}

}  // namespace

cudaError_t batch16_configure() {
    const int c = cudaSharedmemCarveoutMaxShared;
    const auto A = cudaFuncAttributePreferredSharedMemoryCarveout;
    cudaError_t e = cudaFuncSetAttribute((const void *)batch16_kernel<kBatch16R>, A, c);
    cudaError_t e1 = cudaFuncSetAttribute((const void *)batch16_kernel<kBatch16RShort>, A, c);
    cudaError_t e2 = cudaFuncSetAttribute((const void *)batch16_reduce_kernel, A, c);
    return e != cudaSuccess ? e : (e1 != cudaSuccess ? e1 : e2);
}

int batch16_resident_warps(int R, int sms, int max_blocks) {
    const int per_sm = std::max(1, R == kBatch16R ? max_blocks16<kBatch16R>() : max_blocks16<kBatch16RShort>());
    int64_t blocks = (int64_t)per_sm * sms;
    if (max_blocks > 0 && max_blocks < blocks) blocks = max_blocks;
    return (int)(blocks * kWarps);
}

cudaError_t batch16_launch(const Batch16Args &a, int R, int sms, int max_blocks, int64_t npacked, BestRec *pbest,
                           cudaStream_t st) {
    if (R != kBatch16R && R != kBatch16RShort) return cudaErrorInvalidValue;
    if (a.nunits > 0) {
        const int per_sm = std::max(1, R == kBatch16R ? max_blocks16<kBatch16R>() : max_blocks16<kBatch16RShort>());
        const int64_t need = (a.nunits + kWarps - 1) / kWarps;
        int64_t limit = (int64_t)per_sm * sms;
        if (max_blocks > 0 && max_blocks < limit) limit = max_blocks;
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(need, limit));
        if (R == kBatch16R) batch16_kernel<kBatch16R><<<blocks, kWarps * 32, 0, st>>>(a);
        else batch16_kernel<kBatch16RShort><<<blocks, kWarps * 32, 0, st>>>(a);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (npacked > 0) {
        const int64_t threads = npacked * 32;
        batch16_reduce_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(a.pairs, npacked, a.ubest, pbest);
        return cudaGetLastError();
    }
    return cudaSuccess;
}

}  // namespace swb
