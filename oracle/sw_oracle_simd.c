/*
 * sw_oracle_simd.c -- AVX-512 restatement of stage 1 (TEST INFRASTRUCTURE ONLY,
 * see sw_oracle.h).  Same contract and same result as orc_stage1_mt(): textbook
 * Gotoh SW (recurrence of src/FindAlignment.cuh:54-56, zero top/left boundaries
 * of src/SWutils.cpp:144-168), best cell chosen by the reference's tie key
 * (orc_tie_key, src/SWkernel.cuh:219-226 + src/SWutils.cpp:286-298) or row-major.
 *
 * It exists so that the oracle can score pairs of 10^13 - 10^14 cells (the
 * chromosome-scale workload) in well under an hour, and it is checked against the
 * scalar orc_stage1() on seeded pairs (tests/test_oracle.py) and against the
 * committed full-matrix golden of the 1 Mbp pair.
 *
 * Layout: the matrix is cut into strips of 16 rows; one AVX-512 vector holds one
 * row per lane, lane l of strip s is row 16 s + l, and at step k lane l computes
 * column k - l (an anti-diagonal).  The cell above a lane's cell was computed by
 * the lane above at the previous step, so H and F move down the vector by one
 * lane per step (valignd), lane 0 taking the row above the strip from a shared
 * row buffer.  Lane 15 writes the strip's bottom row back into that buffer (in
 * place: it writes column k - 15 after column k was read).  Strips are dealt to
 * threads round robin; a strip waits, per block of columns, until the strip
 * above has written that block.
 *
 * Cells at or above the thread's best score take a scalar path that evaluates
 * the tie key of each such lane, as the scalar oracle does for every cell.
 */
#define _GNU_SOURCE
#include "sw_oracle.h"

#include <immintrin.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

enum { SX_LANES = 16, SX_CW = 4096 };

typedef struct {
    const uint8_t *a;
    int64_t m, n;
    const int32_t *bw;            /* cols as int32, bw[k] for k < n, -2 beyond (never matches) */
    orc_scoring sc;
    orc_geom g;
    int tie;
    int64_t nstrips, nblocks;
    int32_t *rowH, *rowF;         /* bottom row of the strip above, per column */
    _Atomic int64_t *progress;    /* per strip: leading blocks fully written   */
    _Atomic int32_t gbest;        /* best score seen by any thread (threshold)  */
    int nthreads;
} sx_shared;

typedef struct {
    int32_t best;
    uint64_t key;
    int64_t r, c;
} sx_best;

typedef struct {
    sx_shared *sh;
    int id;
    int32_t best;                 /* best score of this thread                     */
    sx_best b[2];                 /* its cell under the tie rule [and row-major]     */
} sx_worker;

static inline void sx_pick(sx_best *b, int32_t h, uint64_t key, int64_t r, int64_t c) {
    if (h > b->best || (h == b->best && key < b->key)) {
        b->best = h;
        b->key = key;
        b->r = r;
        b->c = c;
    }
}

static inline void sx_consider(sx_worker *w, const sx_shared *S, int32_t h, int64_t r, int64_t c) {
    if (S->tie == ORC_TIE_BOTH) {
        sx_pick(&w->b[0], h, orc_tie_key(&S->g, ORC_TIE_REFERENCE, r, c), r, c);
        sx_pick(&w->b[1], h, orc_tie_key(&S->g, ORC_TIE_ROWMAJOR, r, c), r, c);
    } else {
        sx_pick(&w->b[0], h, orc_tie_key(&S->g, S->tie, r, c), r, c);
    }
    if (h > w->best) w->best = h;
}

__attribute__((target("avx512f,avx512bw,avx512vl")))
static void *sx_run(void *arg) {
    sx_worker *w = (sx_worker *)arg;
    sx_shared *S = w->sh;
    const int64_t m = S->m, n = S->n;
    const __m512i vext = _mm512_set1_epi32(S->sc.gap_extend);
    const __m512i vopen = _mm512_set1_epi32(S->sc.gap_open);
    const __m512i vmt = _mm512_set1_epi32(S->sc.match);
    const __m512i vmm = _mm512_set1_epi32(S->sc.mismatch);
    const __m512i vzero = _mm512_setzero_si512();
    const __m512i vlane = _mm512_setr_epi32(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15);
    int32_t hv[SX_LANES];
    for (int64_t s = w->id; s < S->nstrips; s += S->nthreads) {
        const int64_t r0 = s * SX_LANES;
        const int64_t nr = (m - r0 < SX_LANES) ? m - r0 : SX_LANES;
        const __mmask16 rowok = (__mmask16)((1u << nr) - 1u);
        const int below = (r0 + SX_LANES < m);   /* a strip below reads this strip's bottom row */
        int32_t av[SX_LANES];
        for (int l = 0; l < SX_LANES; ++l) av[l] = l < nr ? (int32_t)S->a[r0 + l] : -1;
        const __m512i va = _mm512_loadu_si512(av);
        __m512i vH = vzero, vE = vzero, vD = vzero, vHn = vzero, vFn = vzero, vB = _mm512_set1_epi32(-2);
        int32_t thr = w->best > 0 ? w->best : 1;
        {
            const int32_t gb = atomic_load_explicit(&S->gbest, memory_order_relaxed);
            if (gb > thr) thr = gb;
        }
        __m512i vthr = _mm512_set1_epi32(thr);
        const int64_t kend = n + SX_LANES - 1;
        int64_t k = 0;
        for (int64_t blk = 0; blk <= S->nblocks; ++blk) {
            /* steps [k, k1): all columns read are in blocks <= blk */
            const int64_t k1 = (blk < S->nblocks) ? ((blk + 1) * SX_CW < n ? (blk + 1) * SX_CW : n) : kend;
            if (s > 0 && blk < S->nblocks) {
                while (atomic_load_explicit(&S->progress[s - 1], memory_order_acquire) < blk + 1)
                    _mm_pause();
            }
            for (; k < k1; ++k) {
                /* rowH/rowF/bw are padded past n, so these are plain broadcast loads */
                const __m512i vU = _mm512_alignr_epi32(vHn, _mm512_set1_epi32(S->rowH[k]), 15);
                const __m512i vUF = _mm512_alignr_epi32(vFn, _mm512_set1_epi32(S->rowF[k]), 15);
                vB = _mm512_alignr_epi32(vB, _mm512_set1_epi32(S->bw[k]), 15);
                const __m512i vF = _mm512_max_epi32(_mm512_add_epi32(vUF, vext), _mm512_add_epi32(vU, vopen));
                const __m512i vEn = _mm512_max_epi32(_mm512_add_epi32(vE, vext), _mm512_add_epi32(vH, vopen));
                const __m512i vs = _mm512_mask_blend_epi32(_mm512_cmpeq_epi32_mask(va, vB), vmm, vmt);
                __m512i vh = _mm512_max_epi32(_mm512_add_epi32(vD, vs), vzero);
                vh = _mm512_max_epi32(vh, _mm512_max_epi32(vEn, vF));
                vD = vU;
                /* lanes with column k - l in [0, n) */
                __mmask16 act = rowok;
                if (k < SX_LANES - 1 || k >= n) {
                    const __m512i vc = _mm512_sub_epi32(_mm512_set1_epi32((int32_t)k), vlane);
                    act &= _mm512_cmpge_epi32_mask(vc, vzero) & _mm512_cmplt_epi32_mask(vc, _mm512_set1_epi32((int32_t)n));
                }
                if (k < SX_LANES - 1) {
                    /* lanes that have not reached column 0 keep the left boundary (0) */
                    const __mmask16 started = (__mmask16)((2u << k) - 1u);
                    vh = _mm512_maskz_mov_epi32(started, vh);
                    vHn = vh;
                    vFn = _mm512_maskz_mov_epi32(started, vF);
                    vE = _mm512_maskz_mov_epi32(started, vEn);
                } else {
                    vHn = vh;
                    vFn = vF;
                    vE = vEn;
                }
                vH = vh;
                const __mmask16 hit = _mm512_mask_cmpge_epi32_mask(act, vh, vthr);
                if (__builtin_expect(hit != 0, 0)) {
                    _mm512_storeu_si512(hv, vh);
                    for (unsigned mk = hit; mk; mk &= mk - 1) {
                        const int l = __builtin_ctz(mk);
                        sx_consider(w, S, hv[l], r0 + l, k - l);
                    }
                    if (w->best > thr) {
                        thr = w->best;
                        int32_t gb = atomic_load_explicit(&S->gbest, memory_order_relaxed);
                        while (gb < thr && !atomic_compare_exchange_weak(&S->gbest, &gb, thr)) {
                        }
                        if (gb > thr) thr = gb;
                        vthr = _mm512_set1_epi32(thr);
                    }
                }
                if (below && k >= SX_LANES - 1 && k - (SX_LANES - 1) < n) {
                    /* lane 15 = the strip's bottom row at column k - 15 */
                    _mm512_mask_storeu_epi32(S->rowH + k - 2 * (SX_LANES - 1), (__mmask16)0x8000, vHn);
                    _mm512_mask_storeu_epi32(S->rowF + k - 2 * (SX_LANES - 1), (__mmask16)0x8000, vFn);
                }
            }
            /* columns < k - 15 are written: blocks [0, that / CW) are complete */
            if (blk < S->nblocks) {
                const int64_t done = k - (SX_LANES - 1);
                const int64_t full = done >= n ? S->nblocks : (done > 0 ? done / SX_CW : 0);
                atomic_store_explicit(&S->progress[s], full, memory_order_release);
            }
        }
        atomic_store_explicit(&S->progress[s], S->nblocks, memory_order_release);
    }
    return NULL;
}

int orc_stage1_simd(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
                    const orc_scoring *sc, int tie, int threads, orc_end *out, int64_t *ns_out) {
    const int nout = (tie == ORC_TIE_BOTH) ? 2 : 1;
    if (m < 0 || n < 0) return -2;
    if (!__builtin_cpu_supports("avx512f") || !__builtin_cpu_supports("avx512bw"))
        return -4;
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    if (m == 0 || n == 0) {
        for (int i = 0; i < nout; ++i) { out[i].score = 0; out[i].row = 0; out[i].col = 0; }
        if (ns_out) *ns_out = 0;
        return 0;
    }
    sx_shared *S = calloc(1, sizeof(sx_shared));
    if (!S) return -3;
    S->a = a; S->m = m; S->n = n; S->sc = *sc;
    /* inputs the reference cannot launch on have no ownership order: orc_tie_key
     * then orders row-major */
    if (orc_geometry(m, n, &S->g) != 0 && tie == ORC_TIE_REFERENCE) tie = ORC_TIE_ROWMAJOR;
    S->tie = tie;
    if (threads < 1) threads = 1;
    S->nthreads = threads;
    S->nstrips = (m + SX_LANES - 1) / SX_LANES;
    S->nblocks = (n + SX_CW - 1) / SX_CW;
    /* the masked stores address 15 entries before the column written; reads run
     * 15 entries past the last column (zeros there) */
    int32_t *rowH = calloc((size_t)n + 2 * SX_LANES, sizeof(int32_t));
    int32_t *rowF = calloc((size_t)n + 2 * SX_LANES, sizeof(int32_t));
    int32_t *bw = malloc(sizeof(int32_t) * ((size_t)n + SX_LANES));
    S->progress = calloc((size_t)S->nstrips, sizeof(_Atomic int64_t));
    sx_worker *W = calloc((size_t)threads, sizeof(sx_worker));
    pthread_t *th = calloc((size_t)threads, sizeof(pthread_t));
    int rc = 0;
    if (!rowH || !rowF || !bw || !S->progress || !W || !th) {
        rc = -3;
        goto done;
    }
    S->rowH = rowH + SX_LANES - 1;
    S->rowF = rowF + SX_LANES - 1;
    for (int64_t c = 0; c < n; ++c) bw[c] = b[c];
    for (int64_t c = n; c < n + SX_LANES; ++c) bw[c] = -2;
    S->bw = bw;
    atomic_store(&S->gbest, 0);
    for (int i = 0; i < threads; ++i) {
        W[i].sh = S;
        W[i].id = i;
        pthread_create(&th[i], NULL, sx_run, &W[i]);
    }
    for (int i = 0; i < threads; ++i) pthread_join(th[i], NULL);
    for (int o = 0; o < nout; ++o) {
        sx_best best = {0, 0, 0, 0};
        for (int i = 0; i < threads; ++i) {
            const sx_best *w = &W[i].b[o];
            if (w->best > best.best || (w->best == best.best && w->best > 0 && w->key < best.key)) best = *w;
        }
        out[o].score = best.best;
        out[o].row = best.best > 0 ? best.r : 0;
        out[o].col = best.best > 0 ? best.c : 0;
    }
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (ns_out) *ns_out = (int64_t)(t1.tv_sec - t0.tv_sec) * 1000000000LL + (t1.tv_nsec - t0.tv_nsec);
done:
    free(rowH); free(rowF); free(bw); free((void *)S->progress); free(W); free(th); free(S);
    return rc;
}
