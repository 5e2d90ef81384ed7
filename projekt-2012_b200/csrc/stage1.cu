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
//     value, read from a per-warp shared-memory ring.
//   * Strips are chained through one L2-resident row buffer `hbuf` of 16-byte
//     entries {H + open, tag, F, tag}, written by the strip above with one
//     vector store and read by the strip below with one vector load (each 8-byte
//     half is a single access, so a matching tag in both halves proves the
//     entry is complete; no fences or counters are needed).  The strip below
//     issues its loads one refill (8 steps) ahead and checks the tags a refill
//     later; a mismatch is re-polled with a bounded wait.
//   * The grid is persistent and cooperative (every warp resident).  Strip s runs
//     on block s mod B, warp (s / B) mod 4, so consecutive strips sit on
//     different SMs and every SM gets the same number of strips (+-1).  (Claiming
//     strips from a counter instead lets the block scheduler crowd some SMs, and
//     the chain of strips then runs at the pace of the most crowded one.)
//   * Substitution score: with at most four distinct column bytes (DNA) a
//     per-column table word holds (s - open) for codes 0..3 and one PRMT with a
//     per-row selector picks the sign-extended score (TAB); otherwise the raw
//     bytes are compared (CMP).
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
#include <algorithm>
#include <climits>

#include "stage1_core.cuh"

namespace swb {

namespace {

template <int R, bool TAB, bool STORES>
__global__ void __launch_bounds__(kWarps * 32, (R <= 16 ? 4 : 2)) stage1_kernel(Stage1Args a) {
    __shared__ int4 ring_all[kWarps][kRing + kStage];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    int4 *ring = ring_all[wib];
    int4 *stage = ring + kRing;
    const int64_t B = gridDim.x;

    Best b;
    init_best(b, a.open);
    int32_t bho = b.ho;
    bool failed = false;
    for (int64_t round = 0; !failed; ++round) {
        const int64_t s = blockIdx.x + B * (wib + kWarps * round);
        if (s >= a.nstrips) break;
        if (a.trace && lane == 0) {
            uint32_t smid;
            asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
            a.trace[3 * s + 2] = (int64_t)smid;
        }
        if (!run_strip<R, TAB, STORES, !STORES>(a, ring, stage, lane, (int32_t)s, &b, bho)) failed = true;
        if (a.trace && lane == 0) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            a.trace[3 * s + 1] = (int64_t)t;
        }
    }
    if (failed && lane == 0) {
        atomicCAS(&a.err[0], kErrNone, kErrTimeout);
        atomicExch(&a.err[1], 1);
    }
    key_best(&b, a.tie, a.r_origin, a.c_origin);
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

// Row codes and column table words for TAB mode; lut maps a byte to its code
// (0..3 for the column alphabet, 7 for every other byte).
__global__ void encode_kernel(const uint8_t *rows, int64_t m, const uint8_t *cols, int64_t n, const uint8_t *lut,
                              uint8_t *rcode, uint32_t *ctab, uint32_t mm4, uint32_t x1) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) rcode[i] = lut[rows[i]];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t q = lut[cols[i]];
        ctab[i] = q < 4 ? (mm4 ^ (x1 << (8 * q))) : mm4;
    }
}

// Byte presence flags of a sequence (for choosing TAB mode).
__global__ void presence_kernel(const uint8_t *seq, int64_t n, uint32_t *flags) {
    __shared__ uint32_t sh[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) sh[seq[i]] = 1;
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (sh[i]) flags[i] = 1;
}

template <int R, bool TAB>
cudaError_t launch_r(Stage1Args &a, const Stage1Plan &p, cudaStream_t st) {
    void *args[] = {&a};
    const void *fn = (p.stores || a.srows || a.scols) ? (const void *)stage1_kernel<R, TAB, true>
                                                      : (const void *)stage1_kernel<R, TAB, false>;
    cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(p.blocks), dim3(kWarps * 32), args, 0, st);
    if (e != cudaSuccess) return e;
    reduce_best_kernel<<<1, 256, 0, st>>>(a.wbest, (int64_t)p.blocks * kWarps, a.best);
    return cudaGetLastError();
}

template <int R, bool TAB>
int max_blocks_r() {
    int nb = 0, ns = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, stage1_kernel<R, TAB, false>, kWarps * 32, 0) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ns, stage1_kernel<R, TAB, true>, kWarps * 32, 0) != cudaSuccess)
        return 0;
    return nb < ns ? nb : ns;
}

}  // namespace

// Every kernel of the library asks for the largest shared-memory carveout.  An
// SM's L1/shared split is fixed while blocks run on it, so a long-running kernel
// that needs little shared memory would otherwise leave its SMs configured with
// a small carveout, and another lane's kernel that needs more (the walker) could
// not be placed beside it until the long kernel ended.
cudaError_t stage1_configure() {
    const int c = cudaSharedmemCarveoutMaxShared;
    const auto A = cudaFuncAttributePreferredSharedMemoryCarveout;
    cudaError_t e = cudaSuccess;
    for (cudaError_t x : {cudaFuncSetAttribute((const void *)stage1_kernel<8, false, false>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<8, true, false>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<14, false, false>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<14, true, false>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<14, false, true>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<14, true, true>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<16, false, false>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<16, true, false>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<32, false, false>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<32, true, false>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<8, false, true>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<8, true, true>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<16, false, true>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<16, true, true>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<32, false, true>, A, c),
                          cudaFuncSetAttribute((const void *)stage1_kernel<32, true, true>, A, c),
                          cudaFuncSetAttribute((const void *)reduce_best_kernel, A, c),
                          cudaFuncSetAttribute((const void *)encode_kernel, A, c),
                          cudaFuncSetAttribute((const void *)presence_kernel, A, c)})
        if (x != cudaSuccess) e = x;
    return e;
}

int stage1_max_blocks_per_sm(int R, bool tab) {
    switch (R) {
        case 8: return tab ? max_blocks_r<8, true>() : max_blocks_r<8, false>();
        case 14: return tab ? max_blocks_r<14, true>() : max_blocks_r<14, false>();
        case 16: return tab ? max_blocks_r<16, true>() : max_blocks_r<16, false>();
        case 32: return tab ? max_blocks_r<32, true>() : max_blocks_r<32, false>();
        default: return 0;
    }
}

Stage1Plan stage1_plan(int64_t m, int64_t n, int device_sms, int R_hint, bool tab) {
    Stage1Plan p;
    p.R = (R_hint == 8 || R_hint == 14 || R_hint == 16 || R_hint == 32) ? R_hint : 16;
    p.tab = tab;
    p.warps_per_block = kWarps;
    p.strip_rows = 32LL * p.R;
    p.nstrips = (m + p.strip_rows - 1) / p.strip_rows;
    const int per_sm = stage1_max_blocks_per_sm(p.R, tab);
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
    if (p.tab) {
        switch (p.R) {
            case 8: return launch_r<8, true>(a, p, st);
            case 14: return launch_r<14, true>(a, p, st);
            case 16: return launch_r<16, true>(a, p, st);
            case 32: return launch_r<32, true>(a, p, st);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (p.R) {
        case 8: return launch_r<8, false>(a, p, st);
        case 14: return launch_r<14, false>(a, p, st);
        case 16: return launch_r<16, false>(a, p, st);
        case 32: return launch_r<32, false>(a, p, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t stage1_presence(const uint8_t *seq, int64_t n, uint32_t *flags, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(flags, 0, 256 * sizeof(uint32_t), st);
    if (e != cudaSuccess || n <= 0) return e;
    int blocks = (int)std::min<int64_t>(1024, (n + 255) / 256);
    presence_kernel<<<blocks, 256, 0, st>>>(seq, n, flags);
    return cudaGetLastError();
}

cudaError_t stage1_encode(const uint8_t *rows, int64_t m, const uint8_t *cols, int64_t n, const uint8_t *d_lut,
                          uint8_t *rcode, uint32_t *ctab, int32_t mt1, int32_t mm1, uint32_t *tab_hi,
                          cudaStream_t st) {
    const uint32_t mmb = (uint32_t)(uint8_t)(int8_t)mm1;
    const uint32_t mm4 = mmb * 0x01010101u;
    const uint32_t x1 = ((uint32_t)(uint8_t)(int8_t)mt1 ^ mmb) & 0xFFu;
    *tab_hi = mm4;
    int blocks = (int)std::min<int64_t>(4096, (std::max(m, n) + 255) / 256);
    if (blocks < 1) blocks = 1;
    encode_kernel<<<blocks, 256, 0, st>>>(rows, m, cols, n, d_lut, rcode, ctab, mm4, x1);
    return cudaGetLastError();
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
