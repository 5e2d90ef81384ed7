// traceback.cu -- stage 2: the alignment (canonical traceback) on the GPU.
//
// Replaces the reference's stage 2 (src/Crosspointer.cpp:104-338 with the
// reverse kernels of src/TraceBack.cuh:7-472 and the host join of
// src/SWutils.cpp:175-231).  The reference searches backwards for crosspoints
// on its special rows; its search hangs or exits on most inputs, so this build
// defines the path directly: the traceback of the forward matrix from the end
// cell with a fixed precedence (in H: diagonal > E (column base against a gap)
// > F (row base against a gap); in E or F: extend > open), and reports the
// reference's crosspoints (the path's last cell on every row X with
// (X + 1) % (4T) == 0, src/Builders.cpp:16) along that path.  The path does not
// depend on any tuning parameter of this build.
//
// How: stage 1 keeps special rows (H, F) every 512 rows and special columns
// (H, E) every 256 columns.  The walker kernel is one persistent CTA: for the
// 512 x 256 block that holds the current cell it recomputes the block up to
// that cell from the stored boundaries, with one direction byte per cell in
// shared memory, then warp 0 walks the path (32 cells per ballot along
// diagonal, row or column runs) until the path leaves the block, and repeats.
// Pairs whose stores would not fit the HBM budget keep a coarser grid (level 1);
// each level-1 cell the path enters is recomputed by the stage-1 kernel on that
// sub-rectangle, which writes the 512 x 256 stores for it (level 2).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "traceback.h"

namespace swb {
namespace tb {

namespace {

constexpr int kBR = 512;          // block rows (= stage-1 strip height at R = 16)
constexpr int kBC = 256;          // block columns (= special-column spacing)
constexpr int kThreads = 128;     // recompute threads
constexpr int kRT = kBR / kThreads;  // rows per recompute thread (4)

enum : uint8_t { SRC_ZERO = 0, SRC_DIAG = 1, SRC_E = 2, SRC_F = 3, BIT_EEXT = 4, BIT_FEXT = 8, BIT_DZERO = 16 };
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
    int32_t rcorner;               // H at (rr0 - 1, cc0 - 1)
    int32_t xp_interval;           // reference special-row spacing (4T)
    char *ops;                     // reversed op stream (end -> start)
    int64_t ops_cap;
    int64_t *xps;                  // reversed crosspoints: 4 int64 each (row, col, score, gap)
    int64_t xp_cap;
    int64_t *st;                   // walker state in/out: see kSt* below
};

// walker state slots
enum { kStR = 0, kStC, kStState, kStNOps, kStSuffix, kStNXp, kStDone, kStErr, kStStartR, kStStartC, kStN };

// H, E, F of the boundary cells around a block (region-relative fetches).
__device__ __forceinline__ int2 top_hf(const WalkArgs &a, int64_t R0, int64_t c) {
    // (H, F) of row R0 - 1 at column c (c >= cc0 - 1 handled by callers)
    if (R0 == 0) return make_int2(0, 0);
    if (R0 == a.rr0) {
        if (c < a.cc0) return make_int2(a.rcorner, 0);
        return a.rtop ? a.rtop[c - a.cc0] : make_int2(0, 0);
    }
    const int64_t q = (R0 - a.rr0) / kBR - 1;
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

// Recomputes block rows [R0, R1] x cols [C0, C1] into dir (row-major, kBC wide).
// Expects stage_block() to have filled `s` (and a barrier after it).
__device__ void recompute(const WalkArgs &a, int64_t R0, int64_t R1, int64_t C0, int64_t C1, uint8_t *dir,
                          int2 (*xchg)[kThreads / 32], const Stage *s) {
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const int64_t w = C1 - C0 + 1;
    const int64_t r0 = R0 + (int64_t)t * kRT;  // my first row
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
    int32_t upH = 0, upF = 0;  // (H, F) from the row above at my current column
    int32_t prevUpH = hdiag0;  // H of the row above at the previous column
    const int64_t steps = w + kThreads - 1;
    for (int64_t k = 0; k < steps; ++k) {
        const int64_t j = k - t;  // my column offset
        const bool act = (j >= 0 && j < w && r0 <= R1);
        if (t == 0 && j >= 0 && j < w) {
            const int2 tv = s->top[j + 1];
            upH = tv.x;
            upF = tv.y;
        }
        int32_t oH = 0, oF = 0;
        if (act) {
            const uint8_t cb = s->cb[j];
            int32_t hd = prevUpH;
            int32_t hu = upH, fu = upF;
#pragma unroll
            for (int i = 0; i < kRT; ++i) {
                if (r0 + i > R1) break;
                const int32_t eext = El[i] + a.ext, eopen = Hl[i] + a.open;
                const int32_t fext = fu + a.ext, fopen = hu + a.open;
                const int32_t e = max(eext, eopen), f = max(fext, fopen);
                const int32_t dg = hd + (ra[i] == cb ? a.match : a.mismatch);
                const int32_t hv = max(max(0, e), max(f, dg));
                uint8_t v = hv == 0 ? SRC_ZERO : (hv == dg ? SRC_DIAG : (hv == e ? SRC_E : SRC_F));
                if (eext == e) v |= BIT_EEXT;
                if (fext == f) v |= BIT_FEXT;
                if (hd == 0) v |= BIT_DZERO;
                dir[(r0 + i - R0) * kBC + j] = v;
                hd = Hl[i];
                Hl[i] = hv;
                El[i] = e;
                hu = hv;
                fu = f;
            }
            oH = hu;
            oF = fu;
        }
        prevUpH = upH;
        // hand (H, F) of my last row to the thread below for the next step; the
        // cross-warp slot alternates between two buffers so one barrier per step
        // orders both the write of step k and the reuse of the slot at step k + 2
        const int32_t sH = __shfl_up_sync(0xffffffffu, oH, 1);
        const int32_t sF = __shfl_up_sync(0xffffffffu, oF, 1);
        int2 *xb = xchg[k & 1];
        if (lane == 31) xb[warp] = make_int2(oH, oF);
        __syncthreads();
        if (t > 0) {
            if (lane == 0) {
                const int2 v = xb[warp - 1];
                upH = v.x;
                upF = v.y;
            } else {
                upH = sH;
                upF = sF;
            }
            if (j + 1 == 0) prevUpH = hdiag0;  // my first column: diagonal from the left boundary
        }
    }
}

// Warp 0 walks the path through the block [R0, R1] x [C0, C1].
__device__ void walk(const WalkArgs &a, int64_t R0, int64_t C0, const uint8_t *dir, const Stage *sg, int64_t *S) {
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
            const uint8_t v = in ? dir[(rr - R0) * kBC + (cc - C0)] : 0;
            const bool ok = in && (v & 3) == SRC_DIAG && !(v & BIT_DZERO);
            const uint32_t bal = __ballot_sync(0xffffffffu, ok);
            const int nrun = (bal == 0xffffffffu) ? 32 : __ffs(~bal) - 1;
            int32_t s = 0;
            if (lane < nrun) s = sg->rb[rr - R0] == sg->cb[cc - C0] ? a.match : a.mismatch;
            // inclusive prefix of s over lanes: suffix after lane i's cell
            int32_t ps = s;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t u = __shfl_up_sync(0xffffffffu, ps, o);
                if (lane >= o) ps += u;
            }
            // crosspoint: moving from (rr, cc) to (rr-1, cc-1) enters row rr-1 from below
            const bool xp = lane < nrun && ((rr - 1 + 1) % X) == 0 && rr - 1 >= 0;
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
            const int32_t tot = __shfl_sync(0xffffffffu, ps, 31);
            nops += nrun;
            suffix += tot;
            nxp += __popc(xbal);
            r -= nrun;
            c -= nrun;
            if (nrun < 32 && r >= R0 && c >= C0) {
                const uint8_t w = dir[(r - R0) * kBC + (c - C0)];
                const int src = w & 3;
                if (src == SRC_DIAG) {  // the start cell
                    if (lane == 0 && nops < a.ops_cap) a.ops[nops] = 'M';
                    nops += 1;
                    suffix += sg->rb[r - R0] == sg->cb[c - C0] ? a.match : a.mismatch;
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
            const uint8_t v = in ? dir[(r - R0) * kBC + (cc - C0)] : 0;
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
            const uint8_t v = in ? dir[(rr - R0) * kBC + (c - C0)] : 0;
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
            const bool xp = lane < nrun && (rr % X) == 0 && rr - 1 >= 0;
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
__device__ void walk_body(const WalkArgs &a, uint8_t *dir, int2 (*xchg)[kThreads / 32], Stage *sg, int64_t *S) {
    if (threadIdx.x < kStN) S[threadIdx.x] = a.st[threadIdx.x];
    __syncthreads();
    for (int guard = 0; guard < (1 << 30); ++guard) {
        const int64_t r = S[kStR], c = S[kStC];
        if (S[kStDone] || S[kStErr] || r < a.rr0 || c < a.cc0) break;
        const int64_t R0 = a.rr0 + ((r - a.rr0) / kBR) * kBR;
        const int64_t C0 = a.cc0 + ((c - a.cc0) / kBC) * kBC;
        stage_block(a, R0, r, C0, c, sg);
        __syncthreads();
        recompute(a, R0, r, C0, c, dir, xchg, sg);
        __syncthreads();
        if (threadIdx.x < 32) walk(a, R0, C0, dir, sg, S);
        __syncthreads();
    }
    if (threadIdx.x < kStN) a.st[threadIdx.x] = S[threadIdx.x];
}

// One CTA walks one region.
__global__ void __launch_bounds__(kThreads) walk_kernel(WalkArgs a) {
    extern __shared__ uint8_t dir[];
    __shared__ int2 xchg[2][kThreads / 32];
    __shared__ Stage sg;
    __shared__ int64_t S[kStN];
    walk_body(a, dir, xchg, &sg, S);
}

// Batched pairs: CTA b walks pairs b, b + gridDim.x, ... (each pair's whole
// matrix is its region).
__global__ void __launch_bounds__(kThreads) walk_batch_kernel(const WalkArgs *args, int64_t n) {
    extern __shared__ uint8_t dir[];
    __shared__ int2 xchg[2][kThreads / 32];
    __shared__ Stage sg;
    __shared__ int64_t S[kStN];
    __shared__ WalkArgs sa;
    for (int64_t p = blockIdx.x; p < n; p += gridDim.x) {
        __syncthreads();
        if (threadIdx.x == 0) sa = args[p];
        __syncthreads();
        walk_body(sa, dir, xchg, &sg, S);
    }
}

}  // namespace

int64_t choose_special_interval(const swb_options &opts, int64_t m, int64_t n) {
    (void)opts;
    (void)m;
    (void)n;
    return kBR;  // stage 1 keeps every strip's bottom row (512 rows at R = 16)
}

Plan plan_for(const swb_options &opts, int64_t m, int64_t n) {
    Plan p;
    const double budget = (double)(opts.hbm_budget_bytes ? opts.hbm_budget_bytes : (64ULL << 30));
    const double direct = 8.0 * ((double)(m / kBR) * (double)n + (double)(n / kBC) * (double)m);
    if (direct <= budget) {
        p.level1 = false;
        p.kr = kBR;
        p.kc = kBC;
        return p;
    }
    // level 1: multiples of the block grid sized to the budget (half rows, half columns)
    p.level1 = true;
    int64_t kr = kBR, kc = kBC;
    while (8.0 * (double)(m / kr) * (double)n > budget / 2) kr *= 2;
    while (8.0 * (double)(n / kc) * (double)m > budget / 2) kc *= 2;
    p.kr = kr;
    p.kc = kc;
    return p;
}

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
    a.rcorner = in.rcorner;
    a.xp_interval = in.xp_interval;
    a.ops = in.ops;
    a.ops_cap = in.ops_cap;
    a.xps = in.xps;
    a.xp_cap = in.xp_cap;
    a.st = in.dstate;
    return a;
}

int walk_region(cudaStream_t st, const WalkInputs &in, int64_t *host_state, std::string &err) {
    const WalkArgs a = to_args(in);
    cudaError_t e;
    const size_t smem = (size_t)kBR * kBC;
    // the attribute is per device: set it on every call (cheap)
    if ((e = cudaFuncSetAttribute(walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
        cudaSuccess) {
        err = std::string("walker attribute: ") + cudaGetErrorString(e);
        return SWB_ECUDA;
    }
    if ((e = cudaMemcpyAsync(in.dstate, host_state, sizeof(int64_t) * kStN, cudaMemcpyHostToDevice, st)) !=
        cudaSuccess) {
        err = std::string("walker state: ") + cudaGetErrorString(e);
        return SWB_ECUDA;
    }
    walk_kernel<<<1, kThreads, smem, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(host_state, in.dstate, sizeof(int64_t) * kStN, cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        err = std::string("walker: ") + cudaGetErrorString(e);
        return SWB_ECUDA;
    }
    if (host_state[kStErr]) {
        err = "walker: inconsistent direction data";
        return SWB_ECUDA;
    }
    return SWB_OK;
}

int walk_batch(cudaStream_t st, int sms, const WalkInputs *in, int64_t n, void *d_args, int64_t *d_states,
               int64_t *host_states, std::string &err) {
    if (n <= 0) return SWB_OK;
    std::vector<WalkArgs> args((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        args[(size_t)i] = to_args(in[i]);
        args[(size_t)i].st = d_states + i * kStN;
    }
    cudaError_t e;
    const size_t smem = (size_t)kBR * kBC;
    const int64_t grid = std::min<int64_t>(n, (int64_t)std::max(1, sms));
    if ((e = cudaFuncSetAttribute(walk_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(d_args, args.data(), sizeof(WalkArgs) * (size_t)n, cudaMemcpyHostToDevice, st)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(d_states, host_states, sizeof(int64_t) * kStN * (size_t)n, cudaMemcpyHostToDevice,
                             st)) != cudaSuccess) {
        err = std::string("batched walker set-up: ") + cudaGetErrorString(e);
        return SWB_ECUDA;
    }
    walk_batch_kernel<<<(unsigned)grid, kThreads, smem, st>>>((const WalkArgs *)d_args, n);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(host_states, d_states, sizeof(int64_t) * kStN * (size_t)n, cudaMemcpyDeviceToHost,
                             st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
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

size_t walk_args_bytes() { return sizeof(WalkArgs); }

int state_slots() { return kStN; }
int slot_r() { return kStR; }
int slot_c() { return kStC; }
int slot_state() { return kStState; }
int slot_nops() { return kStNOps; }
int slot_nxp() { return kStNXp; }
int slot_done() { return kStDone; }
int slot_start_r() { return kStStartR; }
int slot_start_c() { return kStStartC; }
int block_rows() { return kBR; }
int block_cols() { return kBC; }

}  // namespace tb
}  // namespace swb
