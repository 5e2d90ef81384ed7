// traceback.cu -- stage 2: the alignment (canonical traceback) on the GPU.
//
// Replaces the reference's stage 2 (src/Crosspointer.cpp:104-338 with the
// reverse kernels of src/TraceBack.cuh:7-472 and the host join of
// src/SWutils.cpp:175-231).  The reference searches backwards for crosspoints
// on its special rows; its search hangs or exits on most inputs, so this library
// defines the path directly: the traceback of the forward matrix from the end
// cell with a fixed precedence (in H: diagonal > E (column base against a gap)
// > F (row base against a gap); in E or F: extend > open), and reports the
// reference's crosspoints (the path's last cell on every row X with
// (X + 1) % (4T) == 0, src/Builders.cpp:16) along that path.  The path does not
// depend on any tuning parameter of this library.
//
// How: stage 1 keeps special rows (H, F) at every strip bottom (every 448 or 512
// rows, the strip height) and special columns (H, E) every 256 columns, so every
// block of that grid (at most 512 x 256) can be recomputed from its stored
// boundaries alone, with one direction byte per cell.
// A block's directions do not depend on the path, so the walker of a single
// pair (walk_region) recomputes a predicted corridor of whole blocks at once,
// one CTA per block across the GPU (the staircase of blocks along the diagonal
// from the current cell, with the blocks above and to the left as margin), and
// then one warp walks the path through them (32 cells per ballot along
// diagonal, row or column runs) until it reaches the start or leaves the
// corridor, where the next round predicts from.  Batches of pairs use one CTA
// per pair that recomputes the blocks on its path on demand.  Inside a CTA the
// block recompute is a pipeline of four warps of 128 rows each, handing rows
// down through shared memory with tagged 64-bit words instead of barriers.
// Pairs whose stores would not fit the HBM budget keep a coarser grid (level 1);
// each level-1 cell the path enters is recomputed by the stage-1 kernel on that
// sub-rectangle, which writes the 512 x 256 stores for it (level 2).
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "batch.h"
#include "traceback.h"

namespace swb {
namespace tb {

namespace {

constexpr int kBR = 512;          // block rows (= stage-1 strip height at R = 16)
constexpr int kBC = 256;          // block columns (= special-column spacing)
constexpr int kThreads = 128;     // recompute threads
constexpr int kRT = kBR / kThreads;  // rows per recompute thread (4)

// Direction byte of a cell: where H comes from (2 bits), whether E and F extend,
// whether the diagonal predecessor's H is 0, and whether the cell's two bases
// match (the walk takes the path's substitution scores from it, so it needs
// no sequence bytes).
enum : uint8_t {
    SRC_ZERO = 0, SRC_DIAG = 1, SRC_E = 2, SRC_F = 3, BIT_EEXT = 4, BIT_FEXT = 8, BIT_DZERO = 16, BIT_MATCH = 32
};
enum : int32_t { ST_H = 0, ST_E = 1, ST_F = 2 };

struct WalkArgs {
    const uint8_t *rows, *cols;
    int64_t m, n;                  // whole matrix
    int32_t match, mismatch, open, ext;
    int32_t score;                 // best score (start of the suffix accounting)
    // stores of the current region: rows [rr0, m) x cols [cc0, n) relative
    const int2 *srows;             // [q][ncols_region] (H, F) of region row (q+1)*512 - 1
    const int2 *scols;             // [q][nrows_region] (H, E) of region col (q+1)*256 - 1
    int64_t rr0, cc0;              // region origin
    int64_t rr1, cc1;              // region end (exclusive) for store indexing
    const int2 *rtop;              // (H, F) of row rr0 - 1 over region cols (nullptr: zero)
    const int2 *rleft;             // (H, E) of col cc0 - 1 over region rows (nullptr: zero)
    int32_t xp_interval;           // reference special-row spacing (4T)
    char *ops;                     // reversed op stream (end -> start)
    int64_t ops_cap;
    int64_t *xps;                  // reversed crosspoints: 4 int64 each (row, col, score, gap)
    int64_t xp_cap;
    int64_t *st;                   // walker state in/out: see kSt* below
    int32_t br;                    // block rows of the region's grid (the special-row spacing), <= kBR
};

// walker state slots
enum { kStR = 0, kStC, kStState, kStNOps, kStSuffix, kStNXp, kStDone, kStErr, kStStartR, kStStartC, kStN };

// H, E, F of the boundary cells around a block (region-relative fetches).
__device__ __forceinline__ int2 top_hf(const WalkArgs &a, int64_t R0, int64_t c) {
    // (H, F) of row R0 - 1 at column c (c >= cc0 - 1 handled by callers)
    if (R0 == 0) return make_int2(0, 0);
    if (R0 == a.rr0) {
        if (c < a.cc0) return make_int2((a.rtop && a.rleft) ? a.rtop[-1].x : 0, 0);  // the corner
        return a.rtop ? a.rtop[c - a.cc0] : make_int2(0, 0);
    }
    const int64_t q = (int32_t)(R0 - a.rr0) / a.br - 1;
    if (c < a.cc0) return make_int2(a.rleft ? a.rleft[R0 - 1 - a.rr0].x : 0, 0);
    return a.srows[q * (a.cc1 - a.cc0) + (c - a.cc0)];
}
__device__ __forceinline__ int2 left_he(const WalkArgs &a, int64_t C0, int64_t r) {
    // (H, E) of column C0 - 1 at row r >= rr0
    if (C0 == 0) return make_int2(0, 0);
    if (C0 == a.cc0) return a.rleft ? a.rleft[r - a.rr0] : make_int2(0, 0);
    const int64_t q = (C0 - a.cc0) / kBC - 1;
    return a.scols[q * (a.rr1 - a.rr0) + (r - a.rr0)];
}

// Block inputs staged in shared memory before a recompute, so that the step loop
// and the walk touch no global memory: the top boundary (H, F) of row R0 - 1 at
// columns C0 - 1 .. C1 (index j + 1), and the row / column bytes of the block.
struct Stage {
    int2 top[kBC + 1];
    uint8_t rb[kBR];
    uint8_t cb[kBC];
};

__device__ void stage_block(const WalkArgs &a, int64_t R0, int64_t R1, int64_t C0, int64_t C1, Stage *s) {
    const int64_t w = C1 - C0 + 1, h = R1 - R0 + 1;
    for (int64_t j = (int64_t)threadIdx.x - 1; j < w; j += blockDim.x) {
        s->top[j + 1] = top_hf(a, R0, C0 + j);
        if (j >= 0) s->cb[j] = a.cols[C0 + j];
    }
    for (int64_t i = threadIdx.x; i < h; i += blockDim.x) s->rb[i] = a.rows[R0 + i];
}

// Direction bytes of one block in global memory, in the recompute's step order so
// that every warp store is one coalesced 128-byte line: word (warp, k, lane)
// holds rows 4t .. 4t + 3 (t = 32 warp + lane) of column k - lane.
constexpr int kSteps = kBC + 31;
constexpr int64_t kBlockWords = (int64_t)(kThreads / 32) * kSteps * 32;
struct GlobalDir {
    uint32_t *d;
    __device__ __forceinline__ uint8_t at(int64_t i, int64_t j) const {
        const int t = (int)(i >> 2), lane = t & 31, warp = t >> 5;
        const int64_t k = j + lane;
        return reinterpret_cast<const uint8_t *>(d + ((int64_t)warp * kSteps + k) * 32 + lane)[i & 3];
    }
    __device__ __forceinline__ void put(int t, int64_t /*j*/, int64_t k, uint32_t word) const {
        d[((int64_t)(t >> 5) * kSteps + k) * 32 + (t & 31)] = word;
    }
};

// The same layout in shared memory (a block's words copied in from GlobalDir).
struct SmemDir {
    const uint32_t *d;
    __device__ __forceinline__ uint8_t at(int64_t i, int64_t j) const {
        const int t = (int)(i >> 2), lane = t & 31, warp = t >> 5;
        const int k = (int)j + lane;
        return reinterpret_cast<const uint8_t *>(d + (warp * kSteps + k) * 32 + lane)[i & 3];
    }
};
constexpr size_t kDirTileBytes = sizeof(uint32_t) * (size_t)kBlockWords;  // 146,944: a multiple of 16

// Hand-off between the warps of a recompute: warp w publishes (H, F) of its last
// row (block row 128 (w + 1) - 1) column by column in bnd[w][j] as two 64-bit
// words {H, gen} and {F, gen}, gen being the recompute's generation; warp w + 1
// reads them as the row above and re-reads until both tags show the current
// generation.  A 64-bit shared access is single-copy atomic, so the tag proves its
// value is current without any fence.
struct Xchg {
    unsigned long long bnd[kThreads / 32 - 1][kBC][2];
    int32_t err;
    uint32_t gen;  // generations used so far by this CTA (tags start at 1; entries start at 0)
};

// Zeroes the hand-off tags and the generation count (once per CTA).
__device__ void xchg_init(Xchg *x) {
    unsigned long long *p = &x->bnd[0][0][0];
    for (int i = threadIdx.x; i < (kThreads / 32 - 1) * kBC * 2; i += blockDim.x) p[i] = 0ULL;
    if (threadIdx.x == 0) {
        x->err = 0;
        x->gen = 0;
    }
}

// Upper bound of a warp's wait for the warp above (SM cycles, about 1 s); the
// writer is a warp of the same CTA, so this only guards against a defect.
constexpr long long kXchgWaitCycles = 2LL * 1000 * 1000 * 1000;

__device__ __forceinline__ unsigned long long pack(int32_t v, uint32_t gen) {
    return ((unsigned long long)gen << 32) | (uint32_t)v;
}
__device__ __forceinline__ unsigned long long ld_shared_volatile(const unsigned long long *p) {
    return *reinterpret_cast<const volatile unsigned long long *>(p);
}

// Waits until entry j of boundary b carries generation gen; returns (H, F).  After
// one wait ran out (x->err set) it no longer waits: the warp finishes its loop on
// whatever values it reads and the caller discards the block.
__device__ __forceinline__ int2 take(Xchg *x, int b, int64_t j, uint32_t gen, bool &fail) {
    if (fail) return make_int2(0, 0);
    unsigned long long h = ld_shared_volatile(&x->bnd[b][j][0]);
    unsigned long long f = ld_shared_volatile(&x->bnd[b][j][1]);
    if ((uint32_t)(h >> 32) != gen || (uint32_t)(f >> 32) != gen) {
        const long long t0 = clock64();
        for (;;) {
            h = ld_shared_volatile(&x->bnd[b][j][0]);
            f = ld_shared_volatile(&x->bnd[b][j][1]);
            if ((uint32_t)(h >> 32) == gen && (uint32_t)(f >> 32) == gen) break;
            if (clock64() - t0 > kXchgWaitCycles) {
                fail = true;
                x->err = 1;
                break;
            }
        }
    }
    return make_int2((int32_t)(uint32_t)h, (int32_t)(uint32_t)f);
}

// Recomputes block rows [R0, R1] x cols [C0, C1] into dir.  Expects
// stage_block() to have filled `s`, x->err zeroed, and a barrier after both;
// `gen` must differ from every earlier recompute of this CTA.  Thread t owns
// rows R0 + 4t .. R0 + 4t + 3: each warp is a 128-row wavefront (lane l computes
// column k - l at step k, rows passed down by shuffles) and the four warps form
// a pipeline through x, so no CTA barrier is needed inside the column loop.
template <class D>
__device__ void recompute(const WalkArgs &a, int64_t R0, int64_t R1, int64_t C0, int64_t C1, const D &dir,
                          Xchg *x, const Stage *s, uint32_t gen) {
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const int64_t w = C1 - C0 + 1;
    const int64_t r0 = R0 + (int64_t)t * kRT;  // my first row
    if (R0 + (int64_t)warp * 32 * kRT > R1) return;  // this warp (and every warp below it) has no rows
    int32_t Hl[kRT], El[kRT];
    uint8_t ra[kRT];
#pragma unroll
    for (int i = 0; i < kRT; ++i) {
        const int64_t r = r0 + i;
        if (r <= R1) {
            const int2 v = left_he(a, C0, r);
            Hl[i] = v.x;
            El[i] = v.y;
            ra[i] = s->rb[r - R0];
        } else {
            Hl[i] = 0;
            El[i] = 0;
            ra[i] = 0;
        }
    }
    // H of the row above my first row at column C0 - 1
    int32_t hdiag0;
    if (t == 0) hdiag0 = s->top[0].x;
    else hdiag0 = (r0 - 1 <= R1) ? left_he(a, C0, r0 - 1).x : 0;
    bool fail = false;
    // warps below the first start with a few columns of slack behind the warp above
    if (warp > 0 && lane == 0) take(x, warp - 1, w - 1 < 15 ? w - 1 : 15, gen, fail);
    __syncwarp();
    int32_t upH = 0, upF = 0;  // (H, F) from the row above at my current column
    int32_t prevUpH = hdiag0;  // H of the row above at the previous column
    const bool publish = (lane == 31) && warp < kThreads / 32 - 1 && (r0 + kRT - 1 <= R1);
    const int64_t steps = w + 31;
    for (int64_t k = 0; k < steps; ++k) {
        const int64_t j = k - lane;  // my column offset
        const bool act = (j >= 0 && j < w && r0 <= R1);
        if (lane == 0 && j < w) {
            const int2 tv = (warp == 0) ? s->top[j + 1] : take(x, warp - 1, j, gen, fail);
            upH = tv.x;
            upF = tv.y;
        }
        int32_t oH = 0, oF = 0;
        if (act) {
            const uint8_t cb = s->cb[j];
            int32_t hd = prevUpH;
            int32_t hu = upH, fu = upF;
            uint32_t word = 0;
#pragma unroll
            for (int i = 0; i < kRT; ++i) {
                if (r0 + i <= R1) {
                    const int32_t eext = El[i] + a.ext, eopen = Hl[i] + a.open;
                    const int32_t fext = fu + a.ext, fopen = hu + a.open;
                    const int32_t e = max(eext, eopen), f = max(fext, fopen);
                    const bool same = ra[i] == cb;
                    const int32_t dg = hd + (same ? a.match : a.mismatch);
                    const int32_t hv = max(max(0, e), max(f, dg));
                    uint32_t v = hv == 0 ? SRC_ZERO : (hv == dg ? SRC_DIAG : (hv == e ? SRC_E : SRC_F));
                    if (same) v |= BIT_MATCH;
                    if (eext == e) v |= BIT_EEXT;
                    if (fext == f) v |= BIT_FEXT;
                    if (hd == 0) v |= BIT_DZERO;
                    word |= v << (8 * i);
                    hd = Hl[i];
                    Hl[i] = hv;
                    El[i] = e;
                    hu = hv;
                    fu = f;
                }
            }
            dir.put(t, j, k, word);
            oH = hu;
            oF = fu;
            if (publish) {
                x->bnd[warp][j][0] = pack(oH, gen);
                x->bnd[warp][j][1] = pack(oF, gen);
            }
        }
        prevUpH = upH;
        // hand (H, F) of my last row to the lane below for the next step
        const int32_t sH = __shfl_up_sync(0xffffffffu, oH, 1);
        const int32_t sF = __shfl_up_sync(0xffffffffu, oF, 1);
        if (lane > 0) {
            upH = sH;
            upF = sF;
            if (j + 1 == 0) prevUpH = hdiag0;  // my first column: diagonal from the left boundary
        }
    }
}

// Warp 0 walks the path through the block [R0, R1] x [C0, C1].
// Row and column indices fit 32 bits (pairs are limited to 2^31 - 64 rows), so
// the crosspoint tests use 32-bit remainders.
template <class D>
__device__ void walk(const WalkArgs &a, int64_t R0, int64_t C0, const D &dir, int64_t *S) {
    const int lane = threadIdx.x & 31;
    int64_t r = S[kStR], c = S[kStC];
    int32_t state = (int32_t)S[kStState];
    int64_t nops = S[kStNOps], suffix = S[kStSuffix], nxp = S[kStNXp];
    const int32_t X = a.xp_interval;
    bool done = false, err = false;
    while (!done && !err && r >= R0 && c >= C0) {
        if (state == ST_H) {
            // run of diagonal moves that are not the start
            const int64_t rr = r - lane, cc = c - lane;
            const bool in = rr >= R0 && cc >= C0;
            const uint8_t v = in ? dir.at(rr - R0, cc - C0) : 0;
            const bool ok = in && (v & 3) == SRC_DIAG && !(v & BIT_DZERO);
            const uint32_t bal = __ballot_sync(0xffffffffu, ok);
            const int nrun = (bal == 0xffffffffu) ? 32 : __ffs(~bal) - 1;
            // inclusive prefix over lanes of the run's substitution scores (the
            // suffix after lane i's cell), from one ballot of the matching cells
            const bool mt = lane < nrun && (v & BIT_MATCH);
            const uint32_t mb = __ballot_sync(0xffffffffu, mt);
            const int nle = min(lane + 1, nrun);
            const int mle = __popc(mb & (0xffffffffu >> (31 - lane)));
            const int32_t ps = mle * a.match + (nle - mle) * a.mismatch;
            // crosspoint: moving from (rr, cc) to (rr-1, cc-1) enters row rr-1 from below
            const bool xp = lane < nrun && rr - 1 >= 0 && ((int32_t)rr % X) == 0;
            const uint32_t xbal = __ballot_sync(0xffffffffu, xp);
            if (xp) {
                const int64_t slot = nxp + __popc(xbal & ((1u << lane) - 1));
                if (slot < a.xp_cap) {
                    int64_t *d = a.xps + 4 * slot;
                    d[0] = rr - 1;
                    d[1] = cc - 1;
                    d[2] = (int64_t)a.score - (suffix + ps);
                    d[3] = 0;
                }
            }
            if (lane < nrun && nops + lane < a.ops_cap) a.ops[nops + lane] = 'M';
            const int32_t tot = __popc(mb) * a.match + (nrun - __popc(mb)) * a.mismatch;
            nops += nrun;
            suffix += tot;
            nxp += __popc(xbal);
            r -= nrun;
            c -= nrun;
            if (nrun < 32 && r >= R0 && c >= C0) {
                const uint8_t w = dir.at(r - R0, c - C0);
                const int src = w & 3;
                if (src == SRC_DIAG) {  // the start cell
                    if (lane == 0 && nops < a.ops_cap) a.ops[nops] = 'M';
                    nops += 1;
                    suffix += (w & BIT_MATCH) ? a.match : a.mismatch;
                    S[kStStartR] = r;
                    S[kStStartC] = c;
                    done = true;
                } else if (src == SRC_E) {
                    state = ST_E;
                } else if (src == SRC_F) {
                    state = ST_F;
                } else {
                    err = true;
                }
            }
        } else if (state == ST_E) {
            // horizontal run: 'I' for every cell until the gap opens
            const int64_t cc = c - lane;
            const bool in = cc >= C0;
            const uint8_t v = in ? dir.at(r - R0, cc - C0) : 0;
            const bool ext = in && (v & BIT_EEXT);
            const uint32_t bal = __ballot_sync(0xffffffffu, ext);
            const uint32_t inb = __ballot_sync(0xffffffffu, in);
            int nrun;                                  // cells consumed
            bool opened;                               // run ended with the gap opening
            const int firstno = (bal == 0xffffffffu) ? 32 : __ffs(~bal) - 1;  // first lane not extending
            if (firstno < 32 && ((inb >> firstno) & 1)) {
                nrun = firstno + 1;
                opened = true;
            } else {
                nrun = min(firstno, __popc(inb));
                opened = false;
            }
            if (lane < nrun && nops + lane < a.ops_cap) a.ops[nops + lane] = 'I';
            nops += nrun;
            suffix += (int64_t)(opened ? nrun - 1 : nrun) * a.ext + (opened ? a.open : 0);
            c -= nrun;
            if (opened) state = ST_H;
        } else {
            // vertical run: 'D' for every cell until the gap opens
            const int64_t rr = r - lane;
            const bool in = rr >= R0;
            const uint8_t v = in ? dir.at(rr - R0, c - C0) : 0;
            const bool ext = in && (v & BIT_FEXT);
            const uint32_t bal = __ballot_sync(0xffffffffu, ext);
            const uint32_t inb = __ballot_sync(0xffffffffu, in);
            const int firstno = (bal == 0xffffffffu) ? 32 : __ffs(~bal) - 1;
            int nrun;
            bool opened;
            if (firstno < 32 && ((inb >> firstno) & 1)) {
                nrun = firstno + 1;
                opened = true;
            } else {
                nrun = min(firstno, __popc(inb));
                opened = false;
            }
            // suffix after lane i's cell: i+1 cells, all ext except an opening cell
            const int64_t cost_i = (int64_t)(lane + 1) * a.ext + ((opened && lane == nrun - 1) ? a.open - a.ext : 0);
            // crosspoint: moving from (rr, c) up to (rr-1, c) enters row rr-1 from below;
            // the cell above is in F if this move extended the gap, else in H
            const bool xp = lane < nrun && rr - 1 >= 0 && ((int32_t)rr % X) == 0;
            const uint32_t xbal = __ballot_sync(0xffffffffu, xp);
            if (xp) {
                const int64_t slot = nxp + __popc(xbal & ((1u << lane) - 1));
                if (slot < a.xp_cap) {
                    int64_t *d = a.xps + 4 * slot;
                    d[0] = rr - 1;
                    d[1] = c;
                    d[2] = (int64_t)a.score - (suffix + cost_i);
                    d[3] = (lane == nrun - 1 && opened) ? 0 : 1;
                }
            }
            if (lane < nrun && nops + lane < a.ops_cap) a.ops[nops + lane] = 'D';
            nops += nrun;
            suffix += (int64_t)(opened ? nrun - 1 : nrun) * a.ext + (opened ? a.open : 0);
            nxp += __popc(xbal);
            r -= nrun;
            if (opened) state = ST_H;
        }
        __syncwarp();
    }
    if (lane == 0) {
        S[kStR] = r;
        S[kStC] = c;
        S[kStState] = state;
        S[kStNOps] = nops;
        S[kStSuffix] = suffix;
        S[kStNXp] = nxp;
        if (done) S[kStDone] = 1;
        if (err) S[kStErr] = 1;
    }
}

// Block after block until the start is reached or the path leaves the region
// [rr0, .) x [cc0, .); the state is read from and written back to a.st.
template <class D>
__device__ void walk_body(const WalkArgs &a, const D &dir, Xchg *xc, Stage *sg, int64_t *S) {
    if (threadIdx.x < kStN) S[threadIdx.x] = a.st[threadIdx.x];
    __syncthreads();
    int guard = 0;
    for (; guard < (1 << 30); ++guard) {
        const int64_t r = S[kStR], c = S[kStC];
        if (S[kStDone] || S[kStErr] || r < a.rr0 || c < a.cc0) break;
        const int64_t R0 = a.rr0 + (int64_t)((int32_t)(r - a.rr0) / a.br) * a.br;
        const int64_t C0 = a.cc0 + ((c - a.cc0) / kBC) * kBC;
        stage_block(a, R0, r, C0, c, sg);
        __syncthreads();
        recompute(a, R0, r, C0, c, dir, xc, sg, xc->gen + (uint32_t)guard + 1u);
        __syncthreads();
        if (xc->err) {
            if (threadIdx.x == 0) S[kStErr] = 1;
            __syncthreads();
            break;
        }
        if (threadIdx.x < 32) walk(a, R0, C0, dir, S);
        __syncthreads();
    }
    if (threadIdx.x < kStN) a.st[threadIdx.x] = S[threadIdx.x];
    __syncthreads();
    if (threadIdx.x == 0) xc->gen += (uint32_t)guard + 1u;  // generations used by this region
}

// Precomputes the direction bytes of whole blocks (R0, C0) = blk[2b], blk[2b + 1]
// of a region into gdir + b * kBlockWords (one CTA per block at a time).  A block
// depends only on the stored boundaries, not on the path, so any set of blocks
// can run at once.
__global__ void __launch_bounds__(kThreads) precompute_kernel(WalkArgs a, const int64_t *blk, int64_t nblk,
                                                              uint32_t *gdir, int32_t *err) {
    __shared__ Xchg xc;
    __shared__ Stage sg;
    xchg_init(&xc);
    uint32_t gen = 0;
    for (int64_t b = blockIdx.x; b < nblk; b += gridDim.x) {
        const int64_t R0 = blk[2 * b], C0 = blk[2 * b + 1];
        const int64_t R1 = min(R0 + a.br - 1, a.rr1 - 1), C1 = min(C0 + kBC - 1, a.cc1 - 1);
        __syncthreads();
        stage_block(a, R0, R1, C0, C1, &sg);
        __syncthreads();
        recompute(a, R0, R1, C0, C1, GlobalDir{gdir + b * kBlockWords}, &xc, &sg, ++gen);
    }
    __syncthreads();
    if (threadIdx.x == 0 && xc.err) atomicExch(err, 1);
}

// Sequence bytes of a block for the walk's diagonal scores.
// One warp walks the path through precomputed blocks: block (bi, bj) of the
// region (relative to rr0, cc0) is slot map[(bi - bi0) * mw + (bj - bj0)] of
// gdir, or absent (-1).  Stops where the path enters an absent block, at the
// start cell or on an error; the state is read from and written back to a.st.
// Waits (bounded) for phase `parity` of the mbarrier at shared address bar.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > kXchgWaitCycles) return false;
    }
}

// The walk of each block reads the block's direction words from shared memory:
// on entering a block the warp copies the part the path can still reach (the
// 128-row chunks at or above the current row, the steps up to the current
// column + 31) from gdir with one bulk asynchronous copy (cp.async.bulk, the
// TMA engine) per chunk, completing on an mbarrier; every step of the walk is
// then a shared-memory read instead of a dependent L2 round trip.  The
// direction bytes carry the match bit, so no sequence bytes are read.
__global__ void __launch_bounds__(32) corridor_walk_kernel(WalkArgs a, const uint32_t *gdir, const int32_t *map,
                                                           int64_t bi0, int64_t bj0, int64_t mh, int64_t mw,
                                                           const int32_t *err) {
    extern __shared__ __align__(16) uint32_t dtile[];  // kBlockWords words
    __shared__ int64_t S[kStN];
    __shared__ __align__(8) uint64_t bar_mem;
    const int lane = threadIdx.x;
    const uint32_t bar = (uint32_t)__cvta_generic_to_shared(&bar_mem);
    if (lane < kStN) S[lane] = a.st[lane];
    if (lane == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (*err) {
        if (lane == 0) S[kStErr] = 1;
        __syncwarp();
    }
    uint32_t phase = 0;
    bool in_flight = false;
    for (;;) {
        const int64_t r = S[kStR], c = S[kStC];
        if (S[kStDone] || S[kStErr] || r < a.rr0 || c < a.cc0) break;
        // region offsets fit 32 bits: 32-bit division
        const int64_t bi = (int32_t)(r - a.rr0) / a.br, bj = (c - a.cc0) / kBC;
        if (bi < bi0 || bi >= bi0 + mh || bj < bj0 || bj >= bj0 + mw) break;
        const int32_t slot = map[(bi - bi0) * mw + (bj - bj0)];
        if (slot < 0) break;
        const int64_t R0 = a.rr0 + bi * a.br, C0 = a.cc0 + bj * kBC;
        const int wmax = (int)((r - R0) >> 7);
        const int kn = (int)(c - C0 + 32 < (int64_t)kSteps ? c - C0 + 32 : (int64_t)kSteps);
        const uint32_t chunk = (uint32_t)kn * 32u * 4u;
        __syncwarp();  // the previous block's reads of dtile are done
        if (lane == 0) {
            const uint32_t *src = gdir + (int64_t)slot * kBlockWords;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                         "r"((uint32_t)(wmax + 1) * chunk)
                         : "memory");
            for (int w = 0; w <= wmax; ++w)
                asm volatile(
                    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                        (uint32_t)__cvta_generic_to_shared(dtile + (int64_t)w * kSteps * 32)),
                    "l"(src + (int64_t)w * kSteps * 32), "r"(chunk), "r"(bar)
                    : "memory");
        }
        in_flight = true;
        const bool ok = __all_sync(0xffffffffu, bar_wait(bar, phase & 1));
        if (!ok) {
            if (lane == 0) S[kStErr] = 1;
            __syncwarp();
            break;
        }
        in_flight = false;
        ++phase;
        __syncwarp();
        walk(a, R0, C0, SmemDir{dtile}, S);
        __syncwarp();
    }
    // A copy still in flight after its wait ran out writes this CTA's shared
    // memory, so the warp waits for it once more before the CTA exits.  It reads
    // at most kBlockWords words of this GPU's own memory and lands in
    // microseconds; every wait of the library is bounded (here about 1 s), and a
    // copy that has not landed after two bounds means the device is failing: the
    // error stays set for the host.
    if (in_flight && !__all_sync(0xffffffffu, bar_wait(bar, phase & 1)) && lane == 0) S[kStErr] = 1;
    __syncwarp();
    if (lane < kStN) a.st[lane] = S[lane];
}

// Batched pairs: CTA b walks pairs b, b + gridDim.x, ... (each pair's whole
// matrix is its region), recomputing the blocks on its path on demand into its
// own region of gdir (kBlockWords words per CTA).
// One CTA per pair at a time, pairs p = blockIdx.x, + gridDim.x, ...
__device__ __forceinline__ void walk_pairs(const WalkArgs *args, int64_t n, uint32_t *gdir) {
    __shared__ Xchg xc;
    __shared__ Stage sg;
    __shared__ int64_t S[kStN];
    __shared__ WalkArgs sa;
    xchg_init(&xc);
    const GlobalDir dir{gdir + (int64_t)blockIdx.x * kBlockWords};
    for (int64_t p = blockIdx.x; p < n; p += gridDim.x) {
        __syncthreads();
        if (threadIdx.x == 0) {
            sa = args[p];
            xc.err = 0;
        }
        __syncthreads();
        walk_body(sa, dir, &xc, &sg, S);
    }
}

__global__ void __launch_bounds__(kThreads) walk_batch_kernel(const WalkArgs *args, int64_t n, uint32_t *gdir) {
    walk_pairs(args, n, gdir);
}

// Graphed batches: every pair's walk starts at the best cell the scoring kernel
// merged into pbest (a pair without a positive score is marked done at once).
__global__ void walk_graph_init_kernel(const GraphHdr *h) {
    const int64_t np = h->npairs;
    WalkArgs *args = (WalkArgs *)h->walk_args;
    int64_t *st = h->walk_states;
    const int32_t open = h->ba.open;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += stride) {
        const BestRec b = h->pbest[p];
        const int32_t score = b.valid ? b.ho - open : 0;
        args[p].score = score;
        int64_t *S = st + p * kStN;
#pragma unroll
        for (int k = 0; k < kStN; ++k) S[k] = 0;
        S[kStR] = b.row;
        S[kStC] = b.col;
        if (score <= 0) S[kStDone] = 1;
    }
}

__global__ void __launch_bounds__(kThreads) walk_graph_kernel(const GraphHdr *h) {
    walk_pairs((const WalkArgs *)h->walk_args, h->npairs, h->walk_dir);
}

}  // namespace

cudaError_t walker_configure() {
    const int c = cudaSharedmemCarveoutMaxShared;
    const auto A = cudaFuncAttributePreferredSharedMemoryCarveout;
    cudaError_t e = cudaSuccess;
    for (cudaError_t x : {cudaFuncSetAttribute((const void *)precompute_kernel, A, c),
                          cudaFuncSetAttribute((const void *)corridor_walk_kernel, A, c),
                          cudaFuncSetAttribute((const void *)corridor_walk_kernel,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDirTileBytes),
                          cudaFuncSetAttribute((const void *)walk_batch_kernel, A, c),
                          cudaFuncSetAttribute((const void *)walk_graph_kernel, A, c)})
        if (x != cudaSuccess) e = x;
    return e;
}

bool spill_placement(uint64_t hbm, uint64_t spill, uint64_t rows_bytes, uint64_t cols_bytes, bool *rows_host,
                     bool *cols_host) {
    *rows_host = *cols_host = false;
    if (rows_bytes + cols_bytes <= hbm) return true;
    if (rows_bytes <= spill && cols_bytes <= hbm) return *rows_host = true;
    if (cols_bytes <= spill && rows_bytes <= hbm) return *cols_host = true;
    if (rows_bytes + cols_bytes <= spill) return *rows_host = *cols_host = true;
    return false;
}

Plan plan_for(const swb_options &opts, int64_t m, int64_t n, int64_t br) {
    Plan p;
    if (br <= 0 || br > kBR || br % 32 != 0) br = kBR;
    const double budget = (double)(opts.hbm_budget_bytes ? opts.hbm_budget_bytes : (64ULL << 30));
    const uint64_t rows_bytes = 8ULL * (uint64_t)(m / br) * (uint64_t)n;
    const uint64_t cols_bytes = 8ULL * (uint64_t)(n / kBC) * (uint64_t)m;
    bool rh = false, ch = false;
    if (spill_placement((uint64_t)budget, opts.host_spill_bytes, rows_bytes, cols_bytes, &rh, &ch)) {
        p.level1 = false;
        p.kr = br;
        p.kc = kBC;
        p.br = br;
        return p;
    }
    p.br = kBR;
    // level 1: multiples of the block grid sized to the budget (half rows, half
    // columns).  The row spacing starts at 3584 = 7 x 512 = 8 x 448 rows, so stage
    // 1 may run 448-row strips as well as 512- or 256-row ones, while each level-1
    // cell is recomputed with 512-row blocks.
    p.level1 = true;
    int64_t kr = 7 * kBR, kc = kBC;
    while (8.0 * (double)(m / kr) * (double)n > budget / 2) kr *= 2;
    while (8.0 * (double)(n / kc) * (double)m > budget / 2) kc *= 2;
    p.kr = kr;
    p.kc = kc;
    return p;
}

// Block rows of a region's grid: in.br, or the full block height when unset.
static int64_t block_rows_of(const WalkInputs &in) { return in.br > 0 && in.br <= kBR ? in.br : kBR; }

static WalkArgs to_args(const WalkInputs &in) {
    WalkArgs a{};
    a.rows = in.rows;
    a.cols = in.cols;
    a.m = in.m;
    a.n = in.n;
    a.match = in.sc.match;
    a.mismatch = in.sc.mismatch;
    a.open = in.sc.gap_open;
    a.ext = in.sc.gap_extend;
    a.score = in.score;
    a.srows = in.srows;
    a.scols = in.scols;
    a.rr0 = in.rr0;
    a.cc0 = in.cc0;
    a.rr1 = in.rr1;
    a.cc1 = in.cc1;
    a.rtop = in.rtop;
    a.rleft = in.rleft;
    a.xp_interval = in.xp_interval;
    a.ops = in.ops;
    a.ops_cap = in.ops_cap;
    a.xps = in.xps;
    a.xp_cap = in.xp_cap;
    a.st = in.dstate;
    a.br = (int32_t)block_rows_of(in);
    return a;
}

// Blocks the path is expected to cross next: the staircase of blocks along the
// diagonal from the current cell toward the region's origin (a local alignment
// of related sequences runs close to a diagonal), with the block above and the
// block to the left of each as margin, in walk order, at most `cap` of them.
static void predict_corridor(const WalkInputs &in, int64_t r, int64_t c, int64_t cap, std::vector<int64_t> &blk,
                             int64_t &bi0, int64_t &bj0, int64_t &mh, int64_t &mw, std::vector<int32_t> &map) {
    const int64_t BR = block_rows_of(in);
    std::vector<std::pair<int64_t, int64_t>> list;
    auto add = [&](int64_t bi, int64_t bj) {
        if (bi < 0 || bj < 0 || (int64_t)list.size() >= cap) return;
        for (size_t q = list.size() >= 8 ? list.size() - 8 : 0; q < list.size(); ++q)
            if (list[q].first == bi && list[q].second == bj) return;
        list.emplace_back(bi, bj);
    };
    int64_t bi = (r - in.rr0) / BR, bj = (c - in.cc0) / kBC;
    add(bi, bj);
    add(bi - 1, bj);
    add(bi, bj - 1);
    while ((int64_t)list.size() < cap) {
        const int64_t R0 = in.rr0 + bi * BR, C0 = in.cc0 + bj * kBC;
        const int64_t d = std::min(r - R0 + 1, c - C0 + 1);
        r -= d;
        c -= d;
        if (r < in.rr0 || c < in.cc0) break;
        bi = (r - in.rr0) / BR;
        bj = (c - in.cc0) / kBC;
        add(bi, bj);
        add(bi - 1, bj);
        add(bi, bj - 1);
    }
    int64_t bmin = INT64_MAX, bmax = -1, cmin = INT64_MAX, cmax = -1;
    for (auto &p : list) {
        bmin = std::min(bmin, p.first);
        bmax = std::max(bmax, p.first);
        cmin = std::min(cmin, p.second);
        cmax = std::max(cmax, p.second);
    }
    bi0 = bmin;
    bj0 = cmin;
    mh = bmax - bmin + 1;
    mw = cmax - cmin + 1;
    map.assign((size_t)(mh * mw), -1);
    blk.resize(2 * list.size());
    for (size_t q = 0; q < list.size(); ++q) {
        int32_t &slot = map[(size_t)((list[q].first - bi0) * mw + (list[q].second - bj0))];
        if (slot < 0) slot = (int32_t)q;
        blk[2 * q] = in.rr0 + list[q].first * BR;
        blk[2 * q + 1] = in.cc0 + list[q].second * kBC;
    }
}

int walk_region(cudaStream_t st, int sms, const WalkInputs &in, int64_t *host_state, const Scratch &scr,
                std::string &err, int32_t *launches) {
    const WalkArgs a = to_args(in);
    cudaError_t e;
    const int64_t cap = 4LL * std::max(1, sms);  // blocks per round: one wave at four CTAs per SM
    uint32_t *gdir = (uint32_t *)scr.ensure(scr.owner, kScrGdir, sizeof(uint32_t) * (size_t)(cap * kBlockWords));
    int64_t *d_blk = (int64_t *)scr.ensure(scr.owner, kScrBlk, sizeof(int64_t) * 2 * (size_t)cap);
    int32_t *d_err = (int32_t *)scr.ensure(scr.owner, kScrWalkErr, sizeof(int32_t));
    if (!gdir || !d_blk || !d_err) {
        err = "walker buffers: out of device memory";
        return SWB_ENOMEM;
    }
    if ((e = cudaMemsetAsync(d_err, 0, sizeof(int32_t), st)) != cudaSuccess ||
        (e = scr.put(scr.owner, in.dstate, host_state, sizeof(int64_t) * kStN)) != cudaSuccess) {
        err = std::string("walker state: ") + cudaGetErrorString(e);
        return SWB_ECUDA;
    }
    std::vector<int64_t> blk;
    std::vector<int32_t> map;
    for (int round = 0; round < (1 << 26); ++round) {
        const int64_t r = host_state[kStR], c = host_state[kStC];
        if (host_state[kStDone] || host_state[kStErr] || r < in.rr0 || c < in.cc0) break;
        int64_t bi0, bj0, mh, mw;
        predict_corridor(in, r, c, cap, blk, bi0, bj0, mh, mw, map);
        const int64_t nblk = (int64_t)blk.size() / 2;
        int32_t *d_map = (int32_t *)scr.ensure(scr.owner, kScrMap, sizeof(int32_t) * map.size());
        if (!d_map) {
            err = "walker buffers: out of device memory";
            return SWB_ENOMEM;
        }
        if ((e = scr.put(scr.owner, d_blk, blk.data(), sizeof(int64_t) * blk.size())) != cudaSuccess ||
            (e = scr.put(scr.owner, d_map, map.data(), sizeof(int32_t) * map.size())) != cudaSuccess) {
            err = std::string("walker corridor: ") + cudaGetErrorString(e);
            return SWB_ECUDA;
        }
        precompute_kernel<<<(unsigned)nblk, kThreads, 0, st>>>(a, d_blk, nblk, gdir, d_err);
        corridor_walk_kernel<<<1, 32, kDirTileBytes, st>>>(a, gdir, d_map, bi0, bj0, mh, mw, d_err);
        *launches += 2;
        if ((e = cudaGetLastError()) != cudaSuccess ||
            (e = scr.get(scr.owner, host_state, in.dstate, sizeof(int64_t) * kStN)) != cudaSuccess) {
            err = std::string("walker: ") + cudaGetErrorString(e);
            return SWB_ECUDA;
        }
        if (host_state[kStR] == r && host_state[kStC] == c && !host_state[kStDone] && !host_state[kStErr]) {
            err = "walker: no progress through the current block";
            return SWB_ECUDA;
        }
    }
    if (host_state[kStErr]) {
        err = "walker: inconsistent direction data";
        return SWB_ECUDA;
    }
    return SWB_OK;
}

int64_t walk_batch_ctas(int sms, int64_t n) { return std::max<int64_t>(1, std::min<int64_t>(n, 8LL * std::max(1, sms))); }
size_t walk_batch_dir_bytes(int sms, int64_t n) {
    return sizeof(uint32_t) * (size_t)kBlockWords * (size_t)walk_batch_ctas(sms, n);
}

int walk_batch(cudaStream_t st, int sms, const WalkInputs *in, int64_t n, void *d_args, int64_t *d_states,
               void *d_dir, int64_t *host_states, const Scratch &scr, std::string &err) {
    if (n <= 0) return SWB_OK;
    std::vector<WalkArgs> args((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        args[(size_t)i] = to_args(in[i]);
        args[(size_t)i].st = d_states + i * kStN;
    }
    cudaError_t e;
    const int64_t grid = walk_batch_ctas(sms, n);
    if ((e = scr.put(scr.owner, d_args, args.data(), sizeof(WalkArgs) * (size_t)n)) != cudaSuccess ||
        (e = scr.put(scr.owner, d_states, host_states, sizeof(int64_t) * kStN * (size_t)n)) != cudaSuccess) {
        err = std::string("batched walker set-up: ") + cudaGetErrorString(e);
        return SWB_ECUDA;
    }
    walk_batch_kernel<<<(unsigned)grid, kThreads, 0, st>>>((const WalkArgs *)d_args, n, (uint32_t *)d_dir);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = scr.get(scr.owner, host_states, d_states, sizeof(int64_t) * kStN * (size_t)n)) != cudaSuccess) {
        err = std::string("batched walker: ") + cudaGetErrorString(e);
        return SWB_ECUDA;
    }
    for (int64_t i = 0; i < n; ++i)
        if (host_states[i * kStN + kStErr] || !host_states[i * kStN + kStDone]) {
            err = "batched walker: inconsistent direction data";
            return SWB_ECUDA;
        }
    return SWB_OK;
}

void pack_walk_args(const WalkInputs *in, int64_t n, int64_t *d_states, void *dst) {
    WalkArgs *out = (WalkArgs *)dst;
    for (int64_t i = 0; i < n; ++i) {
        WalkArgs a = to_args(in[i]);
        a.st = d_states + i * kStN;
        std::memcpy(out + i, &a, sizeof a);
    }
}

cudaError_t walk_graph_enqueue(const GraphHdr *d_hdr, int sms, int64_t max_pairs, cudaStream_t st) {
    const int64_t p = std::max<int64_t>(1, max_pairs);
    walk_graph_init_kernel<<<(unsigned)std::min<int64_t>(std::max(1, sms), (p + 255) / 256), 256, 0, st>>>(d_hdr);
    walk_graph_kernel<<<(unsigned)std::min<int64_t>(walk_graph_ctas(sms), p), kThreads, 0, st>>>(d_hdr);
    return cudaGetLastError();
}

int64_t walk_graph_ctas(int sms) { return 8LL * std::max(1, sms); }

size_t walk_args_bytes() { return sizeof(WalkArgs); }

int state_slots() { return kStN; }
int slot_r() { return kStR; }
int slot_c() { return kStC; }
int slot_state() { return kStState; }
int slot_nops() { return kStNOps; }
int slot_nxp() { return kStNXp; }
int slot_done() { return kStDone; }
int slot_err() { return kStErr; }
int slot_start_r() { return kStStartR; }
int slot_start_c() { return kStStartC; }
int block_rows() { return kBR; }
int block_cols() { return kBC; }

}  // namespace tb
}  // namespace swb
