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
//   * Strips are chained through one L2-resident row buffer `hbuf` of 16-byte
//     entries {H + open, tag, F, tag}, written by the strip above with one
//     vector store and read by the strip below with one vector load (each 8-byte
//     half is a single access, so a matching tag in both halves proves the
//     entry is complete; no fences or counters are needed).  The strip below
//     issues its loads one refill ahead and checks the tags a refill later; a
//     mismatch is re-polled with a bounded wait.
//   * The grid is persistent and cooperative (every warp resident).  Strip s runs
//     on block s mod B, warp (s / B) mod 4, so consecutive strips sit on
//     different SMs and every SM gets the same number of strips (+-1).
//   * Optional outputs: special rows (H, F) every `sr_every` strips (the strip's
//     bottom row) and special columns (H, E) every `sc_every` columns.
//   * Optional inputs (traceback recompute of a sub-rectangle): the row above
//     (H, F), the column to the left (H, E) and the corner H.
//
// Recurrence per cell (exact int32, src/FindAlignment.cuh:54-56), written on
// HO = H + open so that the vertical (F) chain is a single DPX op per row:
//     E   = max(E_left + ext, HO_left)                       __viaddmax_s32
//     t   = max(HO_diag + (s - open), E, 0)                  __viaddmax_s32_relu
//     HO  = max(F + open, t + open)                           __viaddmax_s32
//     F'  = max(F + max(ext, open), t + open)  (F of the row below)
// which equals H = max(0, E, F, H_diag + s), F' = max(F + ext, H + open).
#include <climits>

#include "swb_internal.h"

namespace swb {

namespace {

constexpr int kCH = 8;         // columns per ring refill
constexpr int kP = 8;          // ring entries for columns [k + kP, k + kP + kCH) are stored at step k
constexpr int kRing = 32;      // ring entries per warp
constexpr int kWarps = 4;      // warps per block
constexpr unsigned long long kWaitLimitNs = 20ULL * 1000 * 1000 * 1000;  // bound of every wait

enum : int32_t { kErrNone = 0, kErrTimeout = 4 };

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ int32_t ld_volatile(const int32_t *p) {
    return *reinterpret_cast<const volatile int32_t *>(p);
}
__device__ __forceinline__ int4 ld_ll(const int4 *p) {
    int4 v;
    asm volatile("ld.volatile.global.v4.s32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p)
                 : "memory");
    return v;
}
__device__ __forceinline__ void st_ll(int4 *p, int32_t ho, int32_t f, int32_t tag) {
    asm volatile("st.volatile.global.v4.s32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(ho), "r"(tag), "r"(f), "r"(tag)
                 : "memory");
}

__device__ __noinline__ uint64_t tie_key(const TieGeom g, int64_t r, int64_t c) {
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

struct Best {
    int32_t ho;
    uint64_t key;
    int64_t row, col;
};

// Rows of `mask` hold the column maximum cm at column j: keep the smallest key.
__device__ __forceinline__ void slow_best(uint32_t mask, int32_t cm, const Stage1Args &a, Best &b,
                                          int64_t row0, int32_t j) {
    while (mask) {
        const int i = __ffs(mask) - 1;
        mask &= mask - 1;
        const int64_t r = row0 + i;
        if (r >= a.m) break;
        const uint64_t key = tie_key(a.tie, a.r_origin + r, (int64_t)a.c_origin + j);
        if (better(cm, key, b.ho, b.key)) {
            b.ho = cm;
            b.key = key;
            b.row = r;
            b.col = j;
        }
    }
}

template <int R>
struct Lane {
    int32_t ra[R];   // row bytes (256 for rows past the end: never equal to a byte)
    int32_t HO[R];   // H + open of the previous column
    int32_t E[R];    // E of the previous column
    int32_t inHO, inF, inB;  // from the lane above: HO of its last row, F of my row 0, column byte
    int32_t hodPrev;         // HO of the row above my row 0 at the previous column
    int32_t hodInit;         // HO of the row above my row 0 left of column 0
};

struct StripCtx {
    int64_t row0;     // first row of this lane
    int32_t strip;    // strip index (also the tag it writes)
    int32_t n;
    bool sr;          // this strip's bottom row is a special row
    int64_t sr_off;   // srows offset of that row
};

// One anti-diagonal step.  PRED: some lanes of the warp are outside [0, n).
template <int R, bool PRED>
__device__ __forceinline__ void step(Lane<R> &L, const Stage1Args &a, Best &b, const int4 *ring, int lane,
                                     const StripCtx &sc, int32_t k) {
    const int32_t j = k - lane;
    const bool act = !PRED || (j >= 0 && j < sc.n);
    const int32_t cb = L.inB;
    int32_t hod = (PRED && j == 0) ? L.hodInit : L.hodPrev;
    int32_t f = L.inF;
    int32_t flast = 0;
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
    }
    int32_t cm = L.HO[0];
#pragma unroll
    for (int i = 1; i + 1 < R; i += 2) cm = __vimax3_s32(cm, L.HO[i], L.HO[i + 1]);
    if (R % 2 == 0) cm = max(cm, L.HO[R - 1]);
    if (act && cm >= b.ho) {
        uint32_t mask = 0;
#pragma unroll
        for (int i = 0; i < R; ++i) mask |= (L.HO[i] == cm ? 1u : 0u) << i;
        slow_best(mask, cm, a, b, sc.row0, j);
    }
    // special column: this lane's rows at column j
    if (a.scols != nullptr && act && ((j + 1) & (a.sc_every - 1)) == 0) {
        int2 *dst = a.scols + (int64_t)((j + 1) / a.sc_every - 1) * a.m + sc.row0;
#pragma unroll
        for (int i = 0; i < R; ++i)
            if (sc.row0 + i < a.m) dst[i] = make_int2(L.HO[i] - a.open, L.E[i]);
    }

    // outputs toward the lane below; lane 31 hands its slot to lane 0
    const int4 rv = ring[(k + 1) & (kRing - 1)];
    const bool last = (lane == 31);
    if (last && act) {
        st_ll(a.hbuf + j, L.HO[R - 1], f, sc.strip);
        if (sc.sr) a.srows[sc.sr_off + j] = make_int2(L.HO[R - 1] - a.open, flast);
    }
    const int32_t oHO = last ? rv.x : L.HO[R - 1];
    const int32_t oF = last ? rv.y : f;
    const int32_t oB = last ? rv.z : cb;
    L.hodPrev = L.inHO;
    const int src = (lane + 31) & 31;
    L.inHO = __shfl_sync(0xffffffffu, oHO, src);
    L.inF = __shfl_sync(0xffffffffu, oF, src);
    L.inB = __shfl_sync(0xffffffffu, oB, src);
}

// Top-boundary entry of column c for the first strip of the rectangle.
__device__ __forceinline__ int4 top_entry(const Stage1Args &a, int32_t c) {
    int4 v;
    if (a.top) {
        const int2 t = a.top[c];
        v.x = t.x + a.open;
        v.y = max(t.y + a.ext, t.x + a.open);
    } else {
        v.x = a.open;  // H = 0 above the first row
        v.y = a.gx;    // F of row 0 = max(0 + ext, 0 + open)
    }
    v.z = (int32_t)a.cols[c];
    v.w = 0;
    return v;
}

// Ring refill at step k (k % kCH == 0): lanes 0..kCH-1 check the entries they
// loaded one refill ago (columns [k+kP, k+kP+kCH)), store them in the ring and
// issue the loads for the next refill.  Returns false on timeout/abort.
__device__ __forceinline__ bool refill(const Stage1Args &a, int4 *ring, int lane, int32_t strip, int32_t n,
                                       int32_t k, int4 &pre) {
    bool ok = true;
    if (lane < kCH) {
        const int32_t c = k + kP + lane;
        if (c < n) {
            int4 v;
            if (strip == 0) {
                v = top_entry(a, c);
            } else {
                v = pre;
                if (v.y != strip - 1 || v.w != strip - 1) {
                    const unsigned long long t0 = global_ns();
                    for (;;) {
                        v = ld_ll(a.hbuf + c);
                        if (v.y == strip - 1 && v.w == strip - 1) break;
                        if (ld_volatile(&a.err[1]) != 0 || global_ns() - t0 > kWaitLimitNs) {
                            ok = false;
                            break;
                        }
                        __nanosleep(32);
                    }
                }
                v.y = v.z;                        // F
                v.z = (int32_t)a.cols[c];
                v.w = 0;
            }
            ring[c & (kRing - 1)] = v;
        }
        const int32_t cn = c + kCH;
        if (strip > 0 && cn < n) pre = ld_ll(a.hbuf + cn);
    }
    const bool all_ok = __all_sync(0xffffffffu, ok);
    __syncwarp();
    return all_ok;
}

template <int R>
__device__ __forceinline__ bool run_strip(const Stage1Args &a, int4 *ring, int lane, int32_t s, Best &b) {
    Lane<R> L;
    StripCtx sc;
    const int64_t H = 32LL * R;
    sc.row0 = (int64_t)s * H + (int64_t)lane * R;
    sc.strip = s;
    sc.n = (int32_t)a.n;
    sc.sr = a.srows != nullptr && ((int64_t)(s + 1) % a.sr_every) == 0 && (int64_t)(s + 1) * H <= a.m;
    sc.sr_off = sc.sr ? ((int64_t)(s + 1) / a.sr_every - 1) * a.n : 0;
#pragma unroll
    for (int i = 0; i < R; ++i) {
        const int64_t r = sc.row0 + i;
        const bool in = r < a.m;
        L.ra[i] = in ? (int32_t)a.rows[r] : 256;
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
    // prologue: ring entries for columns [0, kP + kCH), prefetch for the first refill
    int4 pre = make_int4(0, 0, 0, 0);
    if (lane < kCH) {
        const int32_t c = kP + kCH + lane;
        if (s > 0 && c < n) pre = ld_ll(a.hbuf + c);
    }
    for (int32_t c0 = 0; c0 < kP + kCH; c0 += kCH) {
        bool ok = true;
        if (lane < kCH && c0 + lane < n) {
            const int32_t c = c0 + lane;
            int4 v;
            if (s == 0) {
                v = top_entry(a, c);
            } else {
                const unsigned long long t0 = global_ns();
                for (;;) {
                    v = ld_ll(a.hbuf + c);
                    if (v.y == s - 1 && v.w == s - 1) break;
                    if (ld_volatile(&a.err[1]) != 0 || global_ns() - t0 > kWaitLimitNs) {
                        ok = false;
                        break;
                    }
                    __nanosleep(64);
                }
                v.y = v.z;
                v.z = (int32_t)a.cols[c];
                v.w = 0;
            }
            ring[c & (kRing - 1)] = v;
        }
        if (!__all_sync(0xffffffffu, ok)) return false;
        __syncwarp();
    }
    {
        const int4 v = ring[0];
        L.inHO = v.x;
        L.inF = v.y;
        L.inB = v.z;
        L.hodPrev = L.hodInit;
    }

    const int32_t kEnd = n + 31;
    const int32_t kA = min(32, kEnd);
    int32_t kB = kA;
    if (n > 32) kB = 32 + ((n - 32) / kCH) * kCH;
    int32_t k = 0;
    // the first refill is at k = 8 (columns [16, 24)); prologue covered [0, 16)
    for (; k < kA; ++k) {
        if (k > 0 && (k % kCH) == 0 && !refill(a, ring, lane, s, n, k, pre)) return false;
        step<R, true>(L, a, b, ring, lane, sc, k);
    }
    for (; k < kB; ++k) {
        if ((k % kCH) == 0 && !refill(a, ring, lane, s, n, k, pre)) return false;
        step<R, false>(L, a, b, ring, lane, sc, k);
    }
    for (; k < kEnd; ++k) {
        if ((k % kCH) == 0 && !refill(a, ring, lane, s, n, k, pre)) return false;
        step<R, true>(L, a, b, ring, lane, sc, k);
    }
    return true;
}

template <int R>
__global__ void __launch_bounds__(kWarps * 32) stage1_kernel(Stage1Args a) {
    __shared__ int4 ring_all[kWarps][kRing];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    int4 *ring = ring_all[wib];
    const int64_t B = gridDim.x;
    const int64_t per_round = B * kWarps;

    Best b;
    b.ho = a.open + 1;  // only H >= 1 is recorded
    b.key = ~0ULL;
    b.row = 0;
    b.col = 0;
    bool failed = false;
    for (int64_t round = 0; !failed; ++round) {
        const int64_t s = blockIdx.x + B * (wib + kWarps * round);
        if (s >= a.nstrips) break;
        (void)per_round;
        if (!run_strip<R>(a, ring, lane, (int32_t)s, b)) failed = true;
    }
    if (failed && lane == 0) {
        atomicCAS(&a.err[0], kErrNone, kErrTimeout);
        atomicExch(&a.err[1], 1);
    }
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
        a.wbest[(int64_t)blockIdx.x * kWarps + wib] = r;
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

template <int R>
cudaError_t launch_r(Stage1Args &a, const Stage1Plan &p, cudaStream_t st) {
    void *args[] = {&a};
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)stage1_kernel<R>, dim3(p.blocks), dim3(kWarps * 32),
                                                args, 0, st);
    if (e != cudaSuccess) return e;
    reduce_best_kernel<<<1, 256, 0, st>>>(a.wbest, (int64_t)p.blocks * kWarps, a.best);
    return cudaGetLastError();
}

template <int R>
int max_blocks_r() {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, stage1_kernel<R>, kWarps * 32, 0) != cudaSuccess) return 0;
    return nb;
}

}  // namespace

int stage1_max_blocks_per_sm(int R, int warps_per_block) {
    (void)warps_per_block;
    switch (R) {
        case 8: return max_blocks_r<8>();
        case 16: return max_blocks_r<16>();
        case 32: return max_blocks_r<32>();
        default: return 0;
    }
}

Stage1Plan stage1_plan(int64_t m, int64_t n, int device_sms, int R_hint) {
    Stage1Plan p;
    p.R = (R_hint == 8 || R_hint == 16 || R_hint == 32) ? R_hint : 32;
    p.warps_per_block = kWarps;
    p.strip_rows = 32LL * p.R;
    p.nstrips = (m + p.strip_rows - 1) / p.strip_rows;
    const int per_sm = stage1_max_blocks_per_sm(p.R, p.warps_per_block);
    const int64_t max_blocks = (int64_t)device_sms * (per_sm > 0 ? per_sm : 1);
    // enough blocks that every strip of the first round has a warp, spread over
    // whole multiples of the SM count when there is room
    int64_t need = (p.nstrips + p.warps_per_block - 1) / p.warps_per_block;
    int64_t blocks = need < max_blocks ? need : max_blocks;
    if (blocks > device_sms && blocks < max_blocks) blocks = ((blocks + device_sms - 1) / device_sms) * device_sms;
    if (blocks > max_blocks) blocks = max_blocks;
    p.blocks = (int)(blocks < 1 ? 1 : blocks);
    (void)n;
    return p;
}

cudaError_t stage1_launch(Stage1Args &a, const Stage1Plan &p, cudaStream_t st) {
    switch (p.R) {
        case 8: return launch_r<8>(a, p, st);
        case 16: return launch_r<16>(a, p, st);
        case 32: return launch_r<32>(a, p, st);
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
