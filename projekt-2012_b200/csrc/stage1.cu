// stage1.cu -- the scoring wavefront (stage 1) for sm_100a.
//
// Replaces the reference's shortPhase/longPhase kernels (src/FindAlignment.cuh:9-278)
// driven by the dk loop of src/main.cu:183-209, plus the special-row dump of
// src/Builders.cpp:27-104 and the best-score reduction of src/SWutils.cpp:286-298.
//
// Layout of the work
//   * A warp owns a strip of 32*R consecutive rows; lane l owns rows
//     [r0 + l*R, r0 + (l+1)*R) and keeps H + open and E of those rows in
//     registers.  At step k lane l computes column j = k - l (anti-diagonal skew
//     of one column per lane), so the (H, F) that lane l-1 produced for its last
//     row at the previous step is exactly the top boundary lane l needs now; it
//     moves by one rotating warp shuffle per value.  Lane 31 turns its shuffle
//     slot around: it sends lane 0 the next column's top boundary and column
//     byte, read from a per-warp shared-memory ring.
//   * Strips are chained through one L2-resident row buffer `hbuf` (n entries):
//     the warp below reads column j of the strip above, then overwrites it with
//     its own bottom row.  Progress counters (st.release / ld.acquire at gpu
//     scope) gate the reads; every wait is bounded and reports SWB_ETIMEOUT.
//   * The grid is persistent and cooperative (every warp resident), warps take
//     strips round-robin, so a strip never waits for a warp that cannot run.
//
// Recurrence per cell (exact int32, src/FindAlignment.cuh:54-56), written on
// HO = H + open so that the vertical (F) chain is a single DPX op per row:
//     E   = max(E_left + ext, HO_left)                       __viaddmax_s32
//     t   = max(HO_diag + (s - open), E, 0)                  __viaddmax_s32_relu
//     HO  = max(F + open, t + open)                           __viaddmax_s32
//     F'  = max(F + max(ext, open), t + open)  (F of the row below)
// which equals H = max(0, E, F, H_diag + s), F' = max(F + ext, H + open).
#include <cooperative_groups.h>
#include <climits>

#include "swb_internal.h"

namespace swb {

namespace {

constexpr int kCH = 8;         // columns per ring refill
constexpr int kP = 16;         // refill lead: columns [k + kP, k + kP + kCH) at step k
constexpr int kRing = 32;      // ring entries per warp (power of two >= kP + kCH)
constexpr unsigned long long kWaitLimitNs = 20ULL * 1000 * 1000 * 1000;  // bound of every wait

enum : int32_t { kErrNone = 0, kErrTimeout = 4 };

__device__ __forceinline__ void st_release(int32_t *p, int32_t v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int32_t ld_acquire(const int32_t *p) {
    int32_t v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ int32_t ld_volatile(const int32_t *p) {
    return *reinterpret_cast<const volatile int32_t *>(p);
}

__device__ __forceinline__ uint64_t tie_key(const TieGeom &g, int64_t r, int64_t c) {
    if (g.mode == kTieRowMajor) return ((uint64_t)r << 32) | (uint64_t)c;
    const int64_t T = g.T, G = g.G, C = g.C;
    const int64_t t = (r >> 2) % T;
    const int64_t s = r / (4 * T);
    const int64_t k = (c + t) / C;
    const int64_t b = G - 1 - (k % G);
    return ((uint64_t)(b * T + t) << 60) | ((uint64_t)(s + k) << 32) |
           ((uint64_t)(c + t - k * C) << 2) | (uint64_t)(r & 3);
}

__device__ __forceinline__ bool better(int32_t ho, uint64_t key, int32_t bho, uint64_t bkey) {
    return ho > bho || (ho == bho && key < bkey);
}

// State of one lane inside a strip.
template <int R>
struct Lane {
    int32_t ra[R];   // row bytes (256 for rows past the end: never equal to a byte)
    int32_t HO[R];   // H + open of the previous column
    int32_t E[R];    // E of the previous column
    int32_t inHO, inF, inB;  // from the lane above: HO of its last row, F of my row 0, column byte
    int32_t hodPrev;         // HO of the row above my row 0 at the previous column
};

struct Best {
    int32_t ho;
    uint64_t key;
    int64_t row, col;
};

template <int R>
__device__ __forceinline__ void slow_best(const Lane<R> &L, const Stage1Args &a, Best &b, int64_t row0,
                                          int64_t j) {
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int32_t h = L.HO[i];
        if (h >= b.ho && row0 + i < a.m) {
            const uint64_t key = tie_key(a.tie, row0 + i, j);
            if (better(h, key, b.ho, b.key)) {
                b.ho = h;
                b.key = key;
                b.row = row0 + i;
                b.col = j;
            }
        }
    }
}

// One anti-diagonal step of the lane.  PRED: some lanes of the warp are
// outside [0, n) and must keep their state.
template <int R, bool PRED>
__device__ __forceinline__ void step(Lane<R> &L, const Stage1Args &a, Best &b, int4 *ring, int lane,
                                     int64_t row0, int64_t k, bool sr_strip, int64_t sr_idx, int32_t strip) {
    const int64_t j = k - lane;
    const bool act = !PRED || (j >= 0 && j < a.n);
    const int32_t cb = L.inB;
    int32_t hod = (PRED && j == 0) ? a.open : L.hodPrev;
    int32_t f = L.inF;
    int32_t flast = 0;
    int32_t cm = INT_MIN;
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int32_t s1 = (L.ra[i] == cb) ? a.mt1 : a.mm1;
        const int32_t e = __viaddmax_s32(L.E[i], a.ext, L.HO[i]);
        const int32_t t = __viaddmax_s32_relu(hod, s1, e);
        const int32_t to = t + a.open;
        const int32_t ho = __viaddmax_s32(f, a.open, to);
        flast = f;
        f = __viaddmax_s32(f, a.gx, to);
        hod = L.HO[i];
        if (act) {
            L.HO[i] = ho;
            L.E[i] = e;
        }
        if ((i & 1) == 1) cm = __vimax3_s32(cm, L.HO[i - 1], L.HO[i]);
    }
    if (R & 1) cm = max(cm, L.HO[R - 1]);
    if (act && cm >= b.ho) slow_best<R>(L, a, b, row0, j);

    // outputs toward the lane below
    int32_t oHO = L.HO[R - 1], oF = f, oB = cb;
    L.hodPrev = L.inHO;
    if (lane == 31) {
        if (act) {
            a.hbuf[j] = make_int2(oHO, oF);
            if (sr_strip) a.srows[sr_idx * a.n + j] = make_int2(oHO - a.open, flast);
            if (((j + 1) % kCH) == 0 || j + 1 == a.n) st_release(&a.progress[strip], (int32_t)(j + 1));
        }
        const int4 v = ring[(k + 1) & (kRing - 1)];
        oHO = v.x;
        oF = v.y;
        oB = v.z;
    }
    const int src = (lane + 31) & 31;
    L.inHO = __shfl_sync(0xffffffffu, oHO, src);
    L.inF = __shfl_sync(0xffffffffu, oF, src);
    L.inB = __shfl_sync(0xffffffffu, oB, src);
}

// Refill ring entries for columns [c0, c0 + kCH) (lanes 0..kCH-1 load one each).
// Returns false on timeout/abort.
__device__ __forceinline__ bool refill(const Stage1Args &a, int4 *ring, int lane, int64_t strip, int64_t c0) {
    if (c0 >= a.n) return true;
    const int64_t c1 = min(a.n, c0 + (int64_t)kCH);
    bool ok = true;
    if (lane < kCH) {
        const int64_t c = c0 + lane;
        if (strip > 0 && ld_acquire(&a.progress[strip - 1]) < (int32_t)c1) {
            const unsigned long long t0 = global_ns();
            while (ld_acquire(&a.progress[strip - 1]) < (int32_t)c1) {
                if (ld_volatile(&a.err[1]) != 0 || global_ns() - t0 > kWaitLimitNs) {
                    ok = false;
                    break;
                }
                __nanosleep(64);
            }
        }
        if (ok && c < a.n) {
            int4 v;
            if (strip > 0) {
                const int2 h = __ldcg(&a.hbuf[c]);
                v.x = h.x;
                v.y = h.y;
            } else {
                v.x = a.open;  // H = 0 above the first row
                v.y = a.gx;    // F of row 0 = max(0 + ext, 0 + open)
            }
            v.z = (int32_t)a.cols[c];
            v.w = 0;
            ring[c & (kRing - 1)] = v;
        }
    }
    const bool all_ok = __all_sync(0xffffffffu, ok);
    __syncwarp();
    return all_ok;
}

template <int R, int WARPS>
__global__ void __launch_bounds__(WARPS * 32) stage1_kernel(Stage1Args a) {
    __shared__ int4 ring_all[WARPS][kRing];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    int4 *ring = ring_all[wib];
    const int64_t gw = (int64_t)blockIdx.x * WARPS + wib;
    const int64_t W = (int64_t)gridDim.x * WARPS;
    const int64_t H = 32LL * R;

    Best b;
    b.ho = a.open + 1;  // only H >= 1 is recorded
    b.key = ~0ULL;
    b.row = 0;
    b.col = 0;
    bool failed = false;

    for (int64_t s = gw; s < a.nstrips && !failed; s += W) {
        Lane<R> L;
        const int64_t row0 = s * H + (int64_t)lane * R;
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const int64_t r = row0 + i;
            L.ra[i] = (r < a.m) ? (int32_t)a.rows[r] : 256;
            L.HO[i] = a.open;  // H = 0 left of column 0
            L.E[i] = 0;        // E = 0 left of column 0 (the reference's zeroed buffer)
        }
        const bool sr_strip = a.srows != nullptr && ((s + 1) % a.sr_every) == 0 && (s + 1) * H <= a.m;
        const int64_t sr_idx = sr_strip ? (s + 1) / a.sr_every - 1 : 0;

        // prologue: columns [0, kP) into the ring, lane 0's inputs for column 0
        for (int64_t c0 = 0; c0 < kP; c0 += kCH) {
            if (!refill(a, ring, lane, s, c0)) { failed = true; break; }
        }
        if (failed) break;
        {
            const int4 v = ring[0];
            L.inHO = v.x;
            L.inF = v.y;
            L.inB = v.z;
            L.hodPrev = a.open;
        }

        const int64_t n = a.n;
        const int64_t kEnd = n + 31;
        const int64_t kA = min((int64_t)32, kEnd);
        int64_t kB = kA;
        if (n > 32) kB = 32 + ((n - 32) / kCH) * kCH;
        int64_t k = 0;
        for (; k < kA && !failed; ++k) {
            if ((k % kCH) == 0 && !refill(a, ring, lane, s, k + kP)) { failed = true; break; }
            step<R, true>(L, a, b, ring, lane, row0, k, sr_strip, sr_idx, (int32_t)s);
        }
        for (; k < kB && !failed; k += kCH) {
            if (!refill(a, ring, lane, s, k + kP)) { failed = true; break; }
#pragma unroll
            for (int u = 0; u < kCH; ++u) step<R, false>(L, a, b, ring, lane, row0, k + u, sr_strip, sr_idx, (int32_t)s);
        }
        for (; k < kEnd && !failed; ++k) {
            if ((k % kCH) == 0 && !refill(a, ring, lane, s, k + kP)) { failed = true; break; }
            step<R, true>(L, a, b, ring, lane, row0, k, sr_strip, sr_idx, (int32_t)s);
        }
    }
    if (failed && lane == 0) {
        atomicCAS(&a.err[0], kErrNone, kErrTimeout);
        atomicExch(&a.err[1], 1);
    }

    // warp reduction of the best cell
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
    if (lane == 0) {
        BestRec r;
        r.ho = b.ho;
        r.valid = (b.key != ~0ULL) ? 1 : 0;
        r.key = b.key;
        r.row = b.row;
        r.col = b.col;
        a.wbest[gw] = r;
    }
}

__global__ void reduce_best_kernel(const BestRec *in, int64_t count, BestRec *out) {
    __shared__ BestRec sh[256];
    BestRec b;
    b.ho = INT_MIN;
    b.valid = 0;
    b.key = ~0ULL;
    b.row = 0;
    b.col = 0;
    for (int64_t i = threadIdx.x; i < count; i += blockDim.x) {
        const BestRec r = in[i];
        if (r.valid && (!b.valid || better(r.ho, r.key, b.ho, b.key))) b = r;
    }
    sh[threadIdx.x] = b;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            const BestRec r = sh[threadIdx.x + w];
            BestRec &m = sh[threadIdx.x];
            if (r.valid && (!m.valid || better(r.ho, r.key, m.ho, m.key))) m = r;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sh[0];
}

template <int R, int WARPS>
cudaError_t launch_r(Stage1Args &a, const Stage1Plan &p, cudaStream_t st) {
    void *args[] = {&a};
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)stage1_kernel<R, WARPS>, dim3(p.blocks),
                                                dim3(WARPS * 32), args, 0, st);
    if (e != cudaSuccess) return e;
    reduce_best_kernel<<<1, 256, 0, st>>>(a.wbest, (int64_t)p.blocks * WARPS, a.best);
    return cudaGetLastError();
}

template <int R, int WARPS>
int max_blocks_r() {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, stage1_kernel<R, WARPS>, WARPS * 32, 0) != cudaSuccess)
        return 0;
    return nb;
}

}  // namespace

int stage1_max_blocks_per_sm(int R, int warps_per_block) {
    (void)warps_per_block;
    switch (R) {
        case 8: return max_blocks_r<8, 4>();
        case 16: return max_blocks_r<16, 4>();
        case 32: return max_blocks_r<32, 4>();
        default: return 0;
    }
}

Stage1Plan stage1_plan(int64_t m, int64_t n, int device_sms, int R_hint) {
    Stage1Plan p;
    p.R = (R_hint == 8 || R_hint == 16 || R_hint == 32) ? R_hint : 16;
    p.warps_per_block = 4;
    p.strip_rows = 32LL * p.R;
    p.nstrips = (m + p.strip_rows - 1) / p.strip_rows;
    const int per_sm = stage1_max_blocks_per_sm(p.R, p.warps_per_block);
    int64_t max_blocks = (int64_t)device_sms * (per_sm > 0 ? per_sm : 1);
    int64_t need = (p.nstrips + p.warps_per_block - 1) / p.warps_per_block;
    p.blocks = (int)(need < max_blocks ? need : max_blocks);
    if (p.blocks < 1) p.blocks = 1;
    (void)n;
    return p;
}

cudaError_t stage1_launch(Stage1Args &a, const Stage1Plan &p, cudaStream_t st) {
    switch (p.R) {
        case 8: return launch_r<8, 4>(a, p, st);
        case 16: return launch_r<16, 4>(a, p, st);
        case 32: return launch_r<32, 4>(a, p, st);
        default: return cudaErrorInvalidValue;
    }
}

uint64_t tie_key_host(const TieGeom &g, int64_t r, int64_t c) {
    if (g.mode == kTieRowMajor) return ((uint64_t)r << 32) | (uint64_t)c;
    const int64_t T = g.T, G = g.G, C = g.C;
    const int64_t t = (r >> 2) % T;
    const int64_t s = r / (4 * T);
    const int64_t k = (c + t) / C;
    const int64_t b = G - 1 - (k % G);
    return ((uint64_t)(b * T + t) << 60) | ((uint64_t)(s + k) << 32) | ((uint64_t)(c + t - k * C) << 2) |
           (uint64_t)(r & 3);
}

}  // namespace swb
