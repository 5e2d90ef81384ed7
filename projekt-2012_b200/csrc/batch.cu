// batch.cu -- the batched scoring wavefront: many independent pairs of uneven
// length in one persistent launch fed from a device work queue.
//
// No counterpart in the reference, which aligns one pair per process
// (src/main.cu:102-249); every pair's recurrence, tie rule and special rows are
// the single-pair ones (stage1_core.cuh), so a pair scores exactly the same
// alone or in a batch.
//
// Work units.  A pair with m rows has ceil(m / 512) strips of 512 rows (16 rows
// per lane).  The host lists every strip of every pair as one work unit, pair
// after pair (longest pairs first, each pair's strips in order), and warps claim
// units from a device counter.  A unit's only dependency is the strip above it,
// which an earlier claim gave to a warp that is already running, so every wait
// ends whether or not the whole grid is resident at once.  A short pair (<= 512 rows) is one unit: one
// warp aligns it alone (inter-sequence mapping).  A longer pair's strips run on
// consecutive warps that pass the strip's bottom row down through the pair's
// tagged row buffer as in the single-pair kernel (intra-sequence wavefront).
//
// Each unit records the best cell of its strip; a second kernel merges the
// strips of each pair (a warp per pair) into the pair's record, which may carry
// the best of strips run by earlier launches (the serving loop runs a pair's
// strips over several launches).
#include <algorithm>
#include <cstdlib>
#include <type_traits>

#include "batch.h"
#include "stage1_core.cuh"

namespace swb {
namespace {

// Store and boundary fields of a pair view: none (score only), per-pair special
// rows and columns (store pass for the traceback), or those plus the top / left
// boundaries of a sub-rectangle (level-1 recompute of the traceback).
struct NoStores {
    static constexpr int2 *srows = nullptr;
    static constexpr int64_t sr_every = 1;
    static constexpr int2 *scols = nullptr;
    static constexpr int32_t sc_every = 1 << 30;
    static constexpr const int2 *top = nullptr;
    static constexpr const int2 *left = nullptr;
    static constexpr int32_t corner = 0;
};
struct WithStores {
    int2 *srows;
    int64_t sr_every;
    int2 *scols;
    int32_t sc_every;
    static constexpr const int2 *top = nullptr;
    static constexpr const int2 *left = nullptr;
    static constexpr int32_t corner = 0;
};
struct WithBounds {
    int2 *srows;
    int64_t sr_every;
    int2 *scols;
    int32_t sc_every;
    const int2 *top;
    const int2 *left;
    int32_t corner;
};

// The argument view the wavefront core reads for one pair of a batch.
template <class S>
struct PairView : S {
    int32_t open, ext, gx, mt1, mm1;
    uint32_t tab_hi;
    int32_t *err;                  // [0] error code, [1] abort flag
    const uint8_t *rows, *cols, *rcode;
    const uint32_t *ctab;
    int64_t m, n;
    int4 *hbuf;
    int32_t *gbest;
    TieGeom tie;
    int64_t wait_limit;
    static constexpr int32_t withhold = 0;
    static constexpr int2 *bottom = nullptr;
    static constexpr int2 *right = nullptr;
    static constexpr int64_t r_origin = 0;
    static constexpr int64_t c_origin = 0;
    static constexpr int64_t *trace = nullptr;
};

// Claims units until the queue is empty and runs each as one strip.
template <int R, bool TAB, class S>
__device__ __forceinline__ void batch_body(const BatchArgs &g) {
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
        const int64_t nunits = g.nunits_dev ? *g.nunits_dev : g.nunits;
        if (u >= nunits || ld_volatile(&g.ctl[2]) != 0) break;
        const BatchPair d = g.pairs[g.unit_pair[u]];
        PairView<S> v;
        v.open = g.open;
        v.ext = g.ext;
        v.gx = g.gx;
        v.mt1 = g.mt1;
        v.mm1 = g.mm1;
        v.tab_hi = g.tab_hi;
        v.err = g.ctl + 1;
        v.rows = g.seq + d.row_off;
        v.cols = g.cseq + d.col_off;
        v.rcode = TAB ? g.rcode + d.row_off : nullptr;
        v.ctab = TAB ? g.ctab + d.col_off : nullptr;
        v.m = d.m;
        v.n = d.n;
        v.hbuf = g.hbuf + d.hbuf_off;
        v.gbest = g.gbest + d.slot;
        v.tie = d.tie;
        v.wait_limit = g.wait_limit;
        if constexpr (!std::is_same<S, NoStores>::value) {
            v.srows = g.srows + d.sr_off;
            v.sr_every = d.sr_every;
            v.scols = g.scols + d.sc_off;
            v.sc_every = d.sc_every;
        }
        if constexpr (std::is_same<S, WithBounds>::value) {
            v.top = d.top;
            v.left = d.left;
            v.corner = (d.top && d.left) ? d.top[-1].x : 0;
        }
        Best b;
        init_best(b, g.open);
        int32_t bho = b.ho;
        const int32_t strip = g.unit_strip ? g.unit_strip[u] : u - d.unit0;
        if (!run_strip<R, TAB, !std::is_same<S, NoStores>::value, false>(v, ring, stage, lane, strip, &b, bho)) {
            if (lane == 0) {
                atomicCAS(&g.ctl[1], kErrNone, kErrTimeout);
                atomicExch(&g.ctl[2], 1);
            }
            break;
        }
        key_best(&b, v.tie, v.r_origin, v.c_origin);
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
            g.ubest[d.ufirst + strip] = r;
        }
    }
}

template <int R, bool TAB, class S>
__global__ void __launch_bounds__(kWarps * 32, (std::is_same<S, NoStores>::value ? 4 : 3)) batch_kernel(BatchArgs g) {
    batch_body<R, TAB, S>(g);
}

// The graphed form: the instance of the other mode returns at once.  The
// arguments stay a kernel parameter, set on the graph when they change (the unit
// count, which changes every call, is read from the header): read from the
// header into registers instead, they cost the step loop 5% (306 vs 290 ms on
// the 100,000-pair batch), because a parameter is a free constant-bank operand
// and the kernel is at its register cap.
template <int R, bool TAB, class S>
__global__ void __launch_bounds__(kWarps * 32, (std::is_same<S, NoStores>::value ? 4 : 3))
    batch_graph_kernel(BatchArgs g, const GraphHdr *h) {
    if ((h->tab != 0) != TAB) return;
    batch_body<R, TAB, S>(g);
}

__device__ __forceinline__ void merge(BestRec &b, const BestRec &r) {
    if (r.valid && (!b.valid || better(r.ho, r.key, b.ho, b.key))) b = r;
}

// Merges the units of pair d of this launch into pbest[d.slot] (one warp).
__device__ __forceinline__ void reduce_pair(const BatchPair &d, int lane, const BestRec *ubest, BestRec *pbest) {
    BestRec b;
    b.ho = INT_MIN;
    b.valid = 0;
    b.key = ~0ULL;
    b.row = 0;
    b.col = 0;
    if (lane == 0) b = pbest[d.slot];
    for (int32_t u = d.ufirst + lane; u < d.ufirst + d.ucount; u += 32) merge(b, ubest[u]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        BestRec o;
        o.ho = __shfl_xor_sync(0xffffffffu, b.ho, off);
        o.valid = __shfl_xor_sync(0xffffffffu, b.valid, off);
        o.key = __shfl_xor_sync(0xffffffffu, b.key, off);
        o.row = __shfl_xor_sync(0xffffffffu, b.row, off);
        o.col = __shfl_xor_sync(0xffffffffu, b.col, off);
        merge(b, o);
    }
    if (lane == 0) pbest[d.slot] = b;
}

// A warp per pair: merges the pair's units of this launch into pbest[slot].
__global__ void batch_reduce_kernel(const BatchPair *pairs, int64_t npairs, const BestRec *ubest, BestRec *pbest) {
    const int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (p >= npairs) return;
    reduce_pair(pairs[p], threadIdx.x & 31, ubest, pbest);
}

__global__ void graph_reduce_kernel(const GraphHdr *h) {
    const int64_t np = h->npairs;
    const BatchPair *pairs = h->ba.pairs;
    const BestRec *ubest = h->ba.ubest;
    BestRec *pbest = h->pbest;
    const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t p = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; p < np; p += warps)
        reduce_pair(pairs[p], threadIdx.x & 31, ubest, pbest);
}

// Graph step 1: resets the launch's control words, per-pair bests and hand-off
// entries, and ORs the byte values of the sequences into the presence bitmap
// (which the decide kernel clears again after reading it).
__global__ void graph_prepare_kernel(const GraphHdr *h) {
    __shared__ uint32_t sh[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int32_t *ctl = h->out;
    if (tid < 4) ctl[tid] = 0;
    int4 *hbuf = h->ba.hbuf;
    for (int64_t i = tid, e = h->hbuf_entries; i < e; i += stride) hbuf[i] = make_int4(-1, -1, -1, -1);
    int32_t *gbest = h->ba.gbest;
    BestRec *pbest = h->pbest;
    for (int64_t i = tid, e = h->npairs; i < e; i += stride) {
        gbest[i] = 0;
        BestRec z;
        z.ho = 0;
        z.valid = 0;
        z.key = 0;
        z.row = 0;
        z.col = 0;
        pbest[i] = z;
    }
    if (h->tab_ok) {
        // 16 bytes per thread and iteration (the sequence section starts 16-byte aligned)
        const uint8_t *seq = h->ba.seq;
        const int64_t nb = h->seq_bytes, nv = nb >> 4;
        const uint4 *v = reinterpret_cast<const uint4 *>(seq);
        for (int64_t i = tid; i < nv; i += stride) {
            const uint4 w = v[i];
            const uint32_t q[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int k = 0; k < 16; ++k) sh[(q[k >> 2] >> (8 * (k & 3))) & 0xFFu] = 1;
        }
        for (int64_t i = (nv << 4) + tid; i < nb; i += stride) sh[seq[i]] = 1;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += blockDim.x)
        if (sh[i]) atomicOr(&h->presence[i >> 5], 1u << (i & 31));
}

// Graph step 2 (one block of 256 threads, thread = byte value): the table path
// when at most four byte values occur; codes in byte order, 7 for absent bytes.
__global__ void graph_decide_kernel(GraphHdr *h) {
    __shared__ uint32_t bits[8];
    const int b = threadIdx.x;
    if (b < 8) bits[b] = h->presence[b];
    __syncthreads();
    if (b < 8) h->presence[b] = 0;
    int total = 0, below = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        total += __popc(bits[k]);
        if (k < (b >> 5)) below += __popc(bits[k]);
    }
    const uint32_t w = bits[b >> 5];
    below += __popc(w & ((1u << (b & 31)) - 1u));
    const bool present = (w >> (b & 31)) & 1u;
    const int tab = (h->tab_ok && total <= 4) ? 1 : 0;
    h->lut[b] = present ? (uint8_t)below : (uint8_t)7;
    if (b == 0) {
        h->tab = tab;
        h->out[4] = tab;
    }
}

// Graph step 3: table encodings of every byte (table path only).
// 16 bytes per thread and iteration; every section of the graph's buffers starts
// 16-byte aligned.
__global__ void graph_encode_kernel(const GraphHdr *h) {
    if (!h->tab) return;
    __shared__ uint8_t lut[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) lut[i] = h->lut[i];
    __syncthreads();
    const uint8_t *seq = h->ba.seq;
    uint8_t *rcode = const_cast<uint8_t *>(h->ba.rcode);
    uint32_t *ctab = const_cast<uint32_t *>(h->ba.ctab);
    const uint32_t mm4 = h->ba.tab_hi, x1 = h->x1;
    const int64_t nb = h->seq_bytes, nv = nb >> 4;
    const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = tid; i < nv; i += stride) {
        const uint4 w = reinterpret_cast<const uint4 *>(seq)[i];
        const uint32_t in[4] = {w.x, w.y, w.z, w.w};
        uint32_t code[4], tw[16];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uint32_t c = 0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const uint32_t q = lut[(in[k] >> (8 * b)) & 0xFFu];
                c |= q << (8 * b);
                tw[4 * k + b] = q < 4 ? (mm4 ^ (x1 << (8 * q))) : mm4;
            }
            code[k] = c;
        }
        reinterpret_cast<uint4 *>(rcode)[i] = make_uint4(code[0], code[1], code[2], code[3]);
        uint4 *ct = reinterpret_cast<uint4 *>(ctab) + 4 * i;
#pragma unroll
        for (int k = 0; k < 4; ++k) ct[k] = make_uint4(tw[4 * k], tw[4 * k + 1], tw[4 * k + 2], tw[4 * k + 3]);
    }
    for (int64_t i = (nv << 4) + tid; i < nb; i += stride) {
        const uint32_t q = lut[seq[i]];
        rcode[i] = (uint8_t)q;
        ctab[i] = q < 4 ? (mm4 ^ (x1 << (8 * q))) : mm4;
    }
}

__global__ void batch_encode_kernel(const uint8_t *seq, int64_t bytes, const uint8_t *lut, uint8_t *rcode,
                                    uint32_t *ctab, uint32_t mm4, uint32_t x1) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < bytes; i += stride) {
        const uint32_t q = lut[seq[i]];
        rcode[i] = (uint8_t)q;
        ctab[i] = q < 4 ? (mm4 ^ (x1 << (8 * q))) : mm4;
    }
}

template <int R, bool TAB, class S>
int max_blocks() {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, batch_kernel<R, TAB, S>, kWarps * 32, 0) != cudaSuccess)
        return 0;
    return nb;
}

template <int R, bool TAB, class S>
cudaError_t launch(const BatchArgs &a, int sms, int cap, cudaStream_t st) {
    const int per_sm = std::max(1, max_blocks<R, TAB, S>());
    const int64_t need = (a.nunits + kWarps - 1) / kWarps;
    int64_t limit = (int64_t)per_sm * sms;
    if (cap > 0 && cap < limit) limit = cap;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(need, limit));
    batch_kernel<R, TAB, S><<<blocks, kWarps * 32, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t batch_configure() {
    const int c = cudaSharedmemCarveoutMaxShared;
    const auto A = cudaFuncAttributePreferredSharedMemoryCarveout;
    cudaError_t e = cudaSuccess;
    for (cudaError_t x : {cudaFuncSetAttribute((const void *)batch_kernel<8, false, NoStores>, A, c),
                          cudaFuncSetAttribute((const void *)batch_kernel<8, true, NoStores>, A, c),
                          cudaFuncSetAttribute((const void *)batch_kernel<16, false, NoStores>, A, c),
                          cudaFuncSetAttribute((const void *)batch_kernel<16, true, NoStores>, A, c),
                          cudaFuncSetAttribute((const void *)batch_kernel<16, false, WithStores>, A, c),
                          cudaFuncSetAttribute((const void *)batch_kernel<16, true, WithStores>, A, c),
                          cudaFuncSetAttribute((const void *)batch_kernel<16, false, WithBounds>, A, c),
                          cudaFuncSetAttribute((const void *)batch_kernel<16, true, WithBounds>, A, c),
                          cudaFuncSetAttribute((const void *)batch_graph_kernel<8, false, NoStores>, A, c),
                          cudaFuncSetAttribute((const void *)batch_graph_kernel<8, true, NoStores>, A, c),
                          cudaFuncSetAttribute((const void *)batch_graph_kernel<16, false, NoStores>, A, c),
                          cudaFuncSetAttribute((const void *)batch_graph_kernel<16, true, NoStores>, A, c),
                          cudaFuncSetAttribute((const void *)batch_graph_kernel<16, false, WithStores>, A, c),
                          cudaFuncSetAttribute((const void *)batch_graph_kernel<16, true, WithStores>, A, c),
                          cudaFuncSetAttribute((const void *)batch_reduce_kernel, A, c),
                          cudaFuncSetAttribute((const void *)batch_encode_kernel, A, c)})
        if (x != cudaSuccess) e = x;
    return e;
}

namespace {

template <int R, bool TAB, class S>
int graph_grid(int sms, int cap) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, batch_graph_kernel<R, TAB, S>, kWarps * 32, 0) != cudaSuccess)
        nb = 1;
    int64_t g = (int64_t)std::max(1, nb) * sms;
    if (cap > 0 && cap < g) g = cap;
    return (int)std::max<int64_t>(1, g);
}

template <int R, class S>
cudaError_t graph_scoring(const GraphHdr *h, int sms, int cap, int64_t max_units, cudaStream_t st) {
    const BatchArgs placeholder{};  // replaced before the first replay
    const int64_t need = std::max<int64_t>(1, (max_units + kWarps - 1) / kWarps);
    const int gt = (int)std::min<int64_t>(graph_grid<R, true, S>(sms, cap), need);
    const int gc = (int)std::min<int64_t>(graph_grid<R, false, S>(sms, cap), need);
    batch_graph_kernel<R, true, S><<<gt, kWarps * 32, 0, st>>>(placeholder, h);
    batch_graph_kernel<R, false, S><<<gc, kWarps * 32, 0, st>>>(placeholder, h);
    return cudaGetLastError();
}

template <int R, class S>
void scoring_funcs(const void **f) {
    f[0] = (const void *)batch_graph_kernel<R, true, S>;
    f[1] = (const void *)batch_graph_kernel<R, false, S>;
}

}  // namespace

cudaError_t batch_graph_enqueue(const GraphHdr *d_hdr, bool traced, int R, int sms, int max_blocks,
                                int64_t max_units, cudaEvent_t ev_mid, cudaStream_t st) {
    // grid-stride kernels: up to 4 blocks of 256 threads per SM, fewer for small batches
    const int wide = (int)std::min<int64_t>(4LL * std::max(1, sms), std::max<int64_t>(std::max(1, sms) / 4, max_units / 8));
    graph_prepare_kernel<<<wide, 256, 0, st>>>(d_hdr);
    graph_decide_kernel<<<1, 256, 0, st>>>(const_cast<GraphHdr *>(d_hdr));
    graph_encode_kernel<<<wide, 256, 0, st>>>(d_hdr);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    if (traced) e = graph_scoring<16, WithStores>(d_hdr, sms, max_blocks, max_units, st);
    else if (R == 8) e = graph_scoring<8, NoStores>(d_hdr, sms, max_blocks, max_units, st);
    else e = graph_scoring<16, NoStores>(d_hdr, sms, max_blocks, max_units, st);
    if (e != cudaSuccess) return e;
    graph_reduce_kernel<<<wide, 256, 0, st>>>(d_hdr);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (ev_mid) e = cudaEventRecordWithFlags(ev_mid, st, cudaEventRecordExternal);
    return e;
}

void batch_graph_scoring_funcs(bool traced, int R, const void **f) {
    if (traced) scoring_funcs<16, WithStores>(f);
    else if (R == 8) scoring_funcs<8, NoStores>(f);
    else scoring_funcs<16, NoStores>(f);
}

int batch_score_rows_per_lane() {
    // measured on the 100,000-pair batch: R = 16 299 ms, R = 8 413 ms
    if (const char *v = std::getenv("SWB_BATCH_R")) {
        const int r = std::atoi(v);
        if (r == 8 || r == 16) return r;
    }
    return 16;
}

int batch_max_blocks_per_sm(bool tab, BatchMode mode) {
    if (mode == kBatchBounds) return tab ? max_blocks<16, true, WithBounds>() : max_blocks<16, false, WithBounds>();
    if (mode == kBatchStores) return tab ? max_blocks<16, true, WithStores>() : max_blocks<16, false, WithStores>();
    return tab ? max_blocks<16, true, NoStores>() : max_blocks<16, false, NoStores>();
}

int batch_resident_warps(bool tab, BatchMode mode, int sms, int max_blocks) {
    int64_t blocks = (int64_t)std::max(1, batch_max_blocks_per_sm(tab, mode)) * sms;
    if (max_blocks > 0 && max_blocks < blocks) blocks = max_blocks;
    return (int)(blocks * kWarps);
}

cudaError_t batch_launch(const BatchArgs &a, bool tab, BatchMode mode, int R, int sms, int max_blocks, int64_t npairs,
                         BestRec *pbest, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    if (a.nunits > 0) {
        if (mode == kBatchBounds)
            e = tab ? launch<16, true, WithBounds>(a, sms, max_blocks, st)
                    : launch<16, false, WithBounds>(a, sms, max_blocks, st);
        else if (mode == kBatchStores)
            e = tab ? launch<16, true, WithStores>(a, sms, max_blocks, st)
                    : launch<16, false, WithStores>(a, sms, max_blocks, st);
        else if (R == 8)
            e = tab ? launch<8, true, NoStores>(a, sms, max_blocks, st) : launch<8, false, NoStores>(a, sms, max_blocks, st);
        else
            e = tab ? launch<16, true, NoStores>(a, sms, max_blocks, st)
                    : launch<16, false, NoStores>(a, sms, max_blocks, st);
        if (e != cudaSuccess) return e;
    }
    if (npairs > 0) {
        const int64_t threads = npairs * 32;
        batch_reduce_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(a.pairs, npairs, a.ubest, pbest);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t batch_encode(const uint8_t *seq, int64_t bytes, const uint8_t *d_lut, uint8_t *rcode, uint32_t *ctab,
                         int32_t mt1, int32_t mm1, uint32_t *tab_hi, cudaStream_t st) {
    const uint32_t mmb = (uint32_t)(uint8_t)(int8_t)mm1;
    const uint32_t mm4 = mmb * 0x01010101u;
    const uint32_t x1 = ((uint32_t)(uint8_t)(int8_t)mt1 ^ mmb) & 0xFFu;
    *tab_hi = mm4;
    if (bytes <= 0) return cudaSuccess;
    const int blocks = (int)std::min<int64_t>(8192, (bytes + 255) / 256);
    batch_encode_kernel<<<blocks, 256, 0, st>>>(seq, bytes, d_lut, rcode, ctab, mm4, x1);
    return cudaGetLastError();
}

}  // namespace swb
