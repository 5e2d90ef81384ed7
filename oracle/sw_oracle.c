/*
 * sw_oracle.c -- CPU restatement of the reference SWalign SW/Gotoh path.
 *
 * TEST INFRASTRUCTURE ONLY (see sw_oracle.h).  Pinned against (1) the golden
 * score/end-cell lines of the reference's Tests/test1.sh ... test5.sh and (2) the
 * reference's own sources compiled for the CPU (oracle/refemu, make ref), on
 * the fixtures and on seeded random pairs (tests/test_oracle.py).
 *
 * What each piece restates:
 *   recurrence     src/FindAlignment.cuh:54-56 (x4 sub-rows :50-98, longPhase twin
 *                  :191-193):  E = max(E_left + ext, H_left + open),
 *                  F = max(F_up + ext, H_up + open),
 *                  H = max(0, E, F, H_diag + (a == b ? match : mismatch)).
 *                  Bytes are compared as they are (no alphabet, FindAlignment.cuh:51).
 *   boundaries     H = E = F = 0 on the top row and left column (the zeroed
 *                  buffers of src/SWutils.cpp:144-168).  Negative E/F values never
 *                  reach H, so H equals textbook Gotoh SW.
 *   shipped carry  (ORC_SHIPPED_CARRY) the shipped kernels keep the left edge of a
 *                  4-row group in vertical-buffer slot (i/4) mod (G*T)
 *                  (src/SWkernel.cuh:108-128, :202-210).  Strips s and s+G share a
 *                  slot, and the wrap in shortPhase (src/FindAlignment.cuh:120-126)
 *                  re-reads the slot without resetting it, so row r >= 4GT starts
 *                  from the (H, E) that row r-4GT had at column P2-t-1 and from the
 *                  H that row r-1-4GT had there (t = (r/4) mod T).  This mode
 *                  reproduces that; it is checked against the reference build.
 *   geometry       launch shape src/SWutils.cpp:233-253 (G=2, T=5 forced; shrunk for
 *                  short inputs); padding src/FASTA.cpp:107-134 ('$' rows to a
 *                  multiple of ceil(len/4), '#' columns to a multiple of ceil(len/G)).
 *   tie rule       per-thread running max with strict '>' in visit order
 *                  (src/FindAlignment.cuh:58-62, :144-149), launches in dk order
 *                  (src/main.cu:183-209), lowest thread index wins in getMaxScore
 *                  (src/SWutils.cpp:286-298); thread/column ownership from getRow /
 *                  getColumn (src/SWkernel.cuh:219-226) and the strip wrap
 *                  (src/FindAlignment.cuh:25-28).  All-zero matrix: score 0 at (0,0).
 */
#define _GNU_SOURCE
#include "sw_oracle.h"

#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static inline int32_t imax(int32_t a, int32_t b) { return a > b ? a : b; }

/* src/FASTA.cpp:107-126: pad to a multiple of C = ceil(len/parts). */
static int64_t pad_len(int64_t len, int64_t parts) {
    if (len <= 0 || parts <= 0) return len;
    int64_t C = (len + parts - 1) / parts;
    if (len % C == 0) return len;
    return len + (C - len % C);
}

int orc_geometry(int64_t rows, int64_t cols, orc_geom *g) {
    int32_t blocks = 2, threads = 5;                       /* SWutils.cpp:239-240 */
    if ((int64_t)threads * blocks * 2 > cols)              /* SWutils.cpp:242-243 */
        blocks = (int32_t)((float)cols / (float)(threads * 2));
    if (blocks == 0) {                                     /* SWutils.cpp:245-248 */
        blocks = 1;
        threads = (int32_t)(cols / 4);
    }
    g->G = blocks;
    g->T = threads;
    g->P1 = pad_len(rows, 4);
    g->P2 = pad_len(cols, blocks);
    g->C = g->P2 / blocks;
    return threads > 0 ? 0 : -1;
}

uint64_t orc_tie_key(const orc_geom *g, int tie, int64_t r, int64_t c) {
    if (tie == ORC_TIE_ROWMAJOR || g->T <= 0)
        return ((uint64_t)r << 32) | (uint64_t)c;
    int64_t T = g->T, G = g->G, C = g->C;
    int64_t t = (r / 4) % T;
    int64_t s = r / (4 * T);
    int64_t k = (c + t) / C;                 /* 0..G; G = finished in the next wrap */
    int64_t b = G - 1 - (k % G);
    uint64_t gidx = (uint64_t)(b * T + t);
    uint64_t step = (uint64_t)(s + k);
    uint64_t inner = (uint64_t)(c + t - k * C);
    uint64_t sub = (uint64_t)(r % 4);
    return (gidx << 60) | (step << 32) | (inner << 2) | sub;
}

int orc_stage1(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
               const orc_scoring *sc, int semantics, int tie, orc_end *out) {
    if (m < 0 || n < 0 || m < n) return -2;
    orc_geom g;
    int ok = orc_geometry(m, n, &g);
    if (ok != 0) {
        if (semantics == ORC_SHIPPED_CARRY) return -1;   /* the reference cannot launch */
        tie = ORC_TIE_ROWMAJOR;
    }
    const int carry = (semantics == ORC_SHIPPED_CARRY);
    const int64_t rows = carry ? g.P1 : m;
    const int64_t cols = carry ? g.P2 : n;
    const int32_t ext = sc->gap_extend, open = sc->gap_open;
    const int32_t mt = sc->match, mm = sc->mismatch;

    int32_t *Hup = calloc((size_t)cols + 1, sizeof(int32_t));
    int32_t *Fup = calloc((size_t)cols + 1, sizeof(int32_t));
    int32_t *cH = NULL, *cE = NULL, *cHd = NULL;
    const int64_t L = 4 * (int64_t)g.G * g.T;
    if (carry) {
        cH = calloc((size_t)rows + 1, sizeof(int32_t));
        cE = calloc((size_t)rows + 1, sizeof(int32_t));
        cHd = calloc((size_t)rows + 1, sizeof(int32_t));
    }
    if (!Hup || !Fup || (carry && (!cH || !cE || !cHd))) {
        free(Hup); free(Fup); free(cH); free(cE); free(cHd);
        return -3;
    }
    int32_t best = 0;
    uint64_t bestkey = 0;
    int64_t br = 0, bc = 0;
    for (int64_t r = 0; r < rows; ++r) {
        const uint8_t ar = r < m ? a[r] : (uint8_t)'$';
        int32_t hl = 0, el = 0, hd = 0;
        int64_t cc = -1, ccn = -1;
        if (carry) {
            if (r >= L) {
                hl = cH[r - L];
                el = cE[r - L];
                hd = (r - 1 - L >= 0) ? cHd[r - 1 - L] : 0;
            }
            cc = g.P2 - ((r / 4) % g.T) - 1;
            ccn = g.P2 - (((r + 1) / 4) % g.T) - 1;
        }
        for (int64_t c = 0; c < cols; ++c) {
            const uint8_t bcv = c < n ? b[c] : (uint8_t)'#';
            const int32_t f = imax(Fup[c] + ext, Hup[c] + open);
            const int32_t e = imax(el + ext, hl + open);
            const int32_t s = (ar == bcv) ? mt : mm;
            const int32_t h = imax(imax(0, e), imax(f, hd + s));
            hd = Hup[c];
            Hup[c] = h;
            Fup[c] = f;
            hl = h;
            el = e;
            if (carry) {
                if (c == cc) { cH[r] = h; cE[r] = e; }
                if (c == ccn) cHd[r] = h;
            }
            if (h >= best && h > 0) {
                const uint64_t key = orc_tie_key(&g, tie, r, c);
                if (h > best || key < bestkey) {
                    best = h;
                    bestkey = key;
                    br = r;
                    bc = c;
                }
            }
        }
    }
    out->score = best;
    out->row = best > 0 ? br : 0;
    out->col = best > 0 ? bc : 0;
    free(Hup); free(Fup); free(cH); free(cE); free(cHd);
    return 0;
}

/* ------------------------------------------------------ multithreaded stage 1 */

typedef struct {
    const uint8_t *a, *b;
    int64_t m, n;
    orc_scoring sc;
    orc_geom g;
    int tie;
    int64_t SH, CW, nstrips, nblocks;
    int32_t *hrowH, *hrowF;          /* bottom row of the last finished strip part */
    _Atomic int64_t *progress;       /* per strip: column blocks finished          */
    int nthreads;
} mt_shared;

typedef struct {
    mt_shared *sh;
    int id;
    int32_t best;
    uint64_t bestkey;
    int64_t br, bc;
} mt_worker;

static void *mt_run(void *arg) {
    mt_worker *w = (mt_worker *)arg;
    mt_shared *S = w->sh;
    const int32_t ext = S->sc.gap_extend, open = S->sc.gap_open;
    const int32_t mt = S->sc.match, mm = S->sc.mismatch;
    int32_t *lH = malloc(sizeof(int32_t) * (size_t)S->SH);
    int32_t *lE = malloc(sizeof(int32_t) * (size_t)S->SH);
    int32_t *upH = malloc(sizeof(int32_t) * (size_t)S->CW);
    int32_t *upF = malloc(sizeof(int32_t) * (size_t)S->CW);
    int32_t best = 0;
    uint64_t bestkey = 0;
    int64_t br = 0, bc = 0;
    for (int64_t s = w->id; s < S->nstrips; s += S->nthreads) {
        const int64_t r0 = s * S->SH;
        const int64_t r1 = (r0 + S->SH < S->m) ? r0 + S->SH : S->m;
        memset(lH, 0, sizeof(int32_t) * (size_t)S->SH);
        memset(lE, 0, sizeof(int32_t) * (size_t)S->SH);
        int32_t corner = 0;                  /* H[r0-1][c0-1] */
        for (int64_t blk = 0; blk < S->nblocks; ++blk) {
            if (s > 0) {
                while (atomic_load_explicit(&S->progress[s - 1], memory_order_acquire) < blk + 1)
                    ;
            }
            const int64_t c0 = blk * S->CW;
            const int64_t c1 = (c0 + S->CW < S->n) ? c0 + S->CW : S->n;
            const int64_t wdt = c1 - c0;
            if (s > 0) {
                memcpy(upH, S->hrowH + c0, sizeof(int32_t) * (size_t)wdt);
                memcpy(upF, S->hrowF + c0, sizeof(int32_t) * (size_t)wdt);
            } else {
                memset(upH, 0, sizeof(int32_t) * (size_t)wdt);
                memset(upF, 0, sizeof(int32_t) * (size_t)wdt);
            }
            const int32_t next_corner = upH[wdt - 1];
            int32_t dcarry = corner;
            for (int64_t r = r0; r < r1; ++r) {
                const uint8_t ar = S->a[r];
                int32_t hl = lH[r - r0], el = lE[r - r0];
                int32_t hd = dcarry;
                dcarry = hl;
                const uint8_t *bp = S->b + c0;
                for (int64_t j = 0; j < wdt; ++j) {
                    const int32_t f = imax(upF[j] + ext, upH[j] + open);
                    const int32_t e = imax(el + ext, hl + open);
                    const int32_t sc = (ar == bp[j]) ? mt : mm;
                    const int32_t h = imax(imax(0, e), imax(f, hd + sc));
                    hd = upH[j];
                    upH[j] = h;
                    upF[j] = f;
                    hl = h;
                    el = e;
                    if (__builtin_expect(h >= best, 0) && h > 0) {
                        const uint64_t key = orc_tie_key(&S->g, S->tie, r, c0 + j);
                        if (h > best || key < bestkey) {
                            best = h;
                            bestkey = key;
                            br = r;
                            bc = c0 + j;
                        }
                    }
                }
                lH[r - r0] = hl;
                lE[r - r0] = el;
            }
            corner = next_corner;
            memcpy(S->hrowH + c0, upH, sizeof(int32_t) * (size_t)wdt);
            memcpy(S->hrowF + c0, upF, sizeof(int32_t) * (size_t)wdt);
            atomic_store_explicit(&S->progress[s], blk + 1, memory_order_release);
        }
    }
    w->best = best;
    w->bestkey = bestkey;
    w->br = br;
    w->bc = bc;
    free(lH); free(lE); free(upH); free(upF);
    return NULL;
}

int orc_stage1_mt(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
                  const orc_scoring *sc, int tie, int threads, orc_end *out, int64_t *ns_out) {
    if (m < 0 || n < 0) return -2;      /* m < n is allowed here (timing samples) */
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    if (m == 0 || n == 0) {
        out->score = 0; out->row = 0; out->col = 0;
        if (ns_out) *ns_out = 0;
        return 0;
    }
    mt_shared S;
    memset(&S, 0, sizeof S);
    S.a = a; S.b = b; S.m = m; S.n = n; S.sc = *sc;
    if (orc_geometry(m, n, &S.g) != 0) tie = ORC_TIE_ROWMAJOR;
    S.tie = tie;
    if (threads < 1) threads = 1;
    S.nthreads = threads;
    S.SH = 64;
    S.CW = 2048;
    S.nstrips = (m + S.SH - 1) / S.SH;
    S.nblocks = (n + S.CW - 1) / S.CW;
    S.hrowH = calloc((size_t)n, sizeof(int32_t));
    S.hrowF = calloc((size_t)n, sizeof(int32_t));
    S.progress = calloc((size_t)S.nstrips, sizeof(_Atomic int64_t));
    mt_worker *W = calloc((size_t)threads, sizeof(mt_worker));
    pthread_t *th = calloc((size_t)threads, sizeof(pthread_t));
    if (!S.hrowH || !S.hrowF || !S.progress || !W || !th) {
        free(S.hrowH); free(S.hrowF); free((void *)S.progress); free(W); free(th);
        return -3;
    }
    for (int i = 0; i < threads; ++i) {
        W[i].sh = &S;
        W[i].id = i;
        pthread_create(&th[i], NULL, mt_run, &W[i]);
    }
    int32_t best = 0;
    uint64_t bestkey = 0;
    int64_t br = 0, bc = 0;
    for (int i = 0; i < threads; ++i) {
        pthread_join(th[i], NULL);
        if (W[i].best > best || (W[i].best == best && W[i].best > 0 && W[i].bestkey < bestkey)) {
            best = W[i].best;
            bestkey = W[i].bestkey;
            br = W[i].br;
            bc = W[i].bc;
        }
    }
    out->score = best;
    out->row = best > 0 ? br : 0;
    out->col = best > 0 ? bc : 0;
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (ns_out) *ns_out = (int64_t)(t1.tv_sec - t0.tv_sec) * 1000000000LL + (t1.tv_nsec - t0.tv_nsec);
    free(S.hrowH); free(S.hrowF); free((void *)S.progress); free(W); free(th);
    return 0;
}

/* --------------------------------------------------------------- special rows */

int64_t orc_special_rows(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
                         const orc_scoring *sc, int64_t k, int32_t *hf, int64_t max_rows) {
    if (k <= 0) return -2;
    const int32_t ext = sc->gap_extend, open = sc->gap_open;
    int32_t *Hup = calloc((size_t)n + 1, sizeof(int32_t));
    int32_t *Fup = calloc((size_t)n + 1, sizeof(int32_t));
    if (!Hup || !Fup) { free(Hup); free(Fup); return -3; }
    int64_t written = 0;
    for (int64_t r = 0; r < m; ++r) {
        int32_t hl = 0, el = 0, hd = 0;
        for (int64_t c = 0; c < n; ++c) {
            const int32_t f = imax(Fup[c] + ext, Hup[c] + open);
            const int32_t e = imax(el + ext, hl + open);
            const int32_t s = (a[r] == b[c]) ? sc->match : sc->mismatch;
            const int32_t h = imax(imax(0, e), imax(f, hd + s));
            hd = Hup[c];
            Hup[c] = h;
            Fup[c] = f;
            hl = h;
            el = e;
        }
        if ((r + 1) % k == 0 && written < max_rows) {
            int32_t *dst = hf + 2 * n * written;
            for (int64_t c = 0; c < n; ++c) {
                dst[2 * c] = Hup[c];
                dst[2 * c + 1] = Fup[c];
            }
            ++written;
        }
    }
    free(Hup); free(Fup);
    return written;
}

/* ------------------------------------------------------------------ traceback */

enum { SRC_ZERO = 0, SRC_DIAG = 1, SRC_E = 2, SRC_F = 3,
       BIT_E_EXT = 4, BIT_F_EXT = 8, BIT_DIAG_ZERO = 16 };

int64_t orc_traceback(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
                      const orc_scoring *sc, int64_t er, int64_t ec,
                      char *ops, int64_t cap, int64_t *sr, int64_t *sc_) {
    return orc_traceback_xp(a, m, b, n, sc, er, ec, ops, cap, sr, sc_, 0, NULL, 0, NULL);
}

int64_t orc_traceback_xp(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
                         const orc_scoring *sc, int64_t er, int64_t ec,
                         char *ops, int64_t cap, int64_t *sr, int64_t *sc_,
                         int64_t xp_interval, int64_t *xps, int64_t xp_cap, int64_t *nxp) {
    if (er < 0 || ec < 0 || er >= m || ec >= n) return -2;
    const int64_t rows = er + 1, cols = ec + 1;       /* the path stays above-left */
    if ((double)rows * (double)cols > 4.0e9) return -1;
    uint8_t *fl = malloc((size_t)rows * (size_t)cols);
    int32_t *Hup = calloc((size_t)cols + 1, sizeof(int32_t));
    int32_t *Fup = calloc((size_t)cols + 1, sizeof(int32_t));
    if (!fl || !Hup || !Fup) { free(fl); free(Hup); free(Fup); return -1; }
    const int32_t ext = sc->gap_extend, open = sc->gap_open;
    int32_t endH = 0;
    for (int64_t r = 0; r < rows; ++r) {
        int32_t hl = 0, el = 0, hd = 0;
        for (int64_t c = 0; c < cols; ++c) {
            const int32_t fext = Fup[c] + ext, fopen = Hup[c] + open;
            const int32_t eext = el + ext, eopen = hl + open;
            const int32_t f = imax(fext, fopen);
            const int32_t e = imax(eext, eopen);
            const int32_t dg = hd + ((a[r] == b[c]) ? sc->match : sc->mismatch);
            const int32_t h = imax(imax(0, e), imax(f, dg));
            uint8_t v;
            if (h == 0) v = SRC_ZERO;
            else if (h == dg) v = SRC_DIAG;
            else if (h == e) v = SRC_E;
            else v = SRC_F;
            if (eext == e) v |= BIT_E_EXT;
            if (fext == f) v |= BIT_F_EXT;
            if (hd == 0) v |= BIT_DIAG_ZERO;
            fl[r * cols + c] = v;
            hd = Hup[c];
            Hup[c] = h;
            Fup[c] = f;
            hl = h;
            el = e;
        }
    }
    endH = Hup[ec];
    free(Hup); free(Fup);
    if (endH <= 0) {
        free(fl);
        *sr = er; *sc_ = ec;
        return 0;
    }
    int64_t r = er, c = ec, k = 0;
    int state = 0;                                    /* 0 = H, 1 = E, 2 = F */
    int64_t ret = -1;
    int64_t suffix = 0, nx = 0;                       /* score of the path after the current cell */
    /* crosspoint: the path's last cell on a row X with (X + 1) % xp_interval == 0,
     * i.e. the cell entered when the walk moves up from row X + 1; its forward
     * value is endH - suffix, gap = 1 when it is entered inside a vertical gap */
#define ORC_XP(rr, cc, gapflag)                                                       \
    do {                                                                              \
        if (xp_interval > 0 && ((rr) + 1) % xp_interval == 0 && (rr) >= 0 && xps) {  \
            if (nx < xp_cap) {                                                        \
                xps[4 * nx] = (rr); xps[4 * nx + 1] = (cc);                           \
                xps[4 * nx + 2] = endH - suffix; xps[4 * nx + 3] = (gapflag);         \
            }                                                                         \
            ++nx;                                                                     \
        }                                                                             \
    } while (0)
    for (;;) {
        if (r < 0 || c < 0) { ret = -2; break; }
        const uint8_t v = fl[r * cols + c];
        if (state == 0) {
            const int src = v & 3;
            if (src == SRC_DIAG) {
                if (k >= cap) { ret = -1; break; }
                ops[k++] = 'M';
                suffix += (a[r] == b[c]) ? sc->match : sc->mismatch;
                if ((v & BIT_DIAG_ZERO) || r == 0 || c == 0) { *sr = r; *sc_ = c; ret = k; break; }
                --r; --c;
                ORC_XP(r, c, 0);
            } else if (src == SRC_E) {
                state = 1;
            } else if (src == SRC_F) {
                state = 2;
            } else { ret = -2; break; }
        } else if (state == 1) {
            if (k >= cap) { ret = -1; break; }
            ops[k++] = 'I';
            suffix += (v & BIT_E_EXT) ? sc->gap_extend : sc->gap_open;
            state = (v & BIT_E_EXT) ? 1 : 0;
            --c;
        } else {
            if (k >= cap) { ret = -1; break; }
            ops[k++] = 'D';
            suffix += (v & BIT_F_EXT) ? sc->gap_extend : sc->gap_open;
            state = (v & BIT_F_EXT) ? 2 : 0;
            --r;
            ORC_XP(r, c, state == 2 ? 1 : 0);
        }
    }
#undef ORC_XP
    if (nxp) *nxp = nx;
    if (xps && nx > 1) {                              /* report top to bottom */
        for (int64_t i = 0, j = (nx < xp_cap ? nx : xp_cap) - 1; i < j; ++i, --j)
            for (int q = 0; q < 4; ++q) {
                int64_t t = xps[4 * i + q]; xps[4 * i + q] = xps[4 * j + q]; xps[4 * j + q] = t;
            }
    }
    free(fl);
    if (ret > 0) {                                    /* reverse to start -> end */
        for (int64_t i = 0, j = ret - 1; i < j; ++i, --j) {
            char t = ops[i]; ops[i] = ops[j]; ops[j] = t;
        }
    }
    return ret;
}

int64_t orc_score_ops(const uint8_t *a, const uint8_t *b, const orc_scoring *sc,
                      int64_t sr, int64_t sc_, const char *ops, int64_t nops) {
    int64_t r = sr, c = sc_, s = 0;
    char prev = 'M';
    /* the recurrence lets a gap run restart through H, so each character after
     * the first costs the better of extend and open */
    const int32_t cont = sc->gap_extend > sc->gap_open ? sc->gap_extend : sc->gap_open;
    for (int64_t i = 0; i < nops; ++i) {
        const char o = ops[i];
        if (o == 'M') {
            s += (a[r] == b[c]) ? sc->match : sc->mismatch;
            ++r; ++c;
        } else if (o == 'I') {
            s += (prev == 'I') ? cont : sc->gap_open;
            ++c;
        } else if (o == 'D') {
            s += (prev == 'D') ? cont : sc->gap_open;
            ++r;
        } else {
            return INT64_MIN;
        }
        prev = o;
    }
    return s;
}

/* Best score of an alignment whose first cell is the diagonal cell (sr, sc_) and
 * whose last cell is (er, ec), with the same gap recurrence as stage 1 but no
 * zero floor: a start cell found by some other search is the start of an optimal
 * local alignment ending at (er, ec) exactly when this equals the best score. */
int64_t orc_anchored_score(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
                           const orc_scoring *sc, int64_t sr, int64_t sc_, int64_t er, int64_t ec) {
    if (sr < 0 || sc_ < 0 || er < sr || ec < sc_ || er >= m || ec >= n) return INT64_MIN;
    const int64_t W = ec - sc_ + 1;
    const int64_t NEG = INT64_MIN / 4;
    int64_t *H = malloc(sizeof(int64_t) * (size_t)W), *F = malloc(sizeof(int64_t) * (size_t)W);
    if (!H || !F) { free(H); free(F); return INT64_MIN; }
    for (int64_t j = 0; j < W; ++j) { H[j] = NEG; F[j] = NEG; }
    for (int64_t i = sr; i <= er; ++i) {
        int64_t hl = NEG, el = NEG, hd = NEG;
        for (int64_t j = 0; j < W; ++j) {
            const int64_t s = (a[i] == b[sc_ + j]) ? sc->match : sc->mismatch;
            const int64_t f = (i > sr) ? (F[j] + sc->gap_extend > H[j] + sc->gap_open ? F[j] + sc->gap_extend
                                                                                      : H[j] + sc->gap_open) : NEG;
            const int64_t e = (j > 0) ? (el + sc->gap_extend > hl + sc->gap_open ? el + sc->gap_extend
                                                                                : hl + sc->gap_open) : NEG;
            int64_t h = (i == sr && j == 0) ? s : hd + s;
            if (e > h) h = e;
            if (f > h) h = f;
            if (h < NEG / 2) h = NEG;
            hd = H[j];
            H[j] = h;
            F[j] = f < NEG / 2 ? NEG : f;
            hl = h;
            el = e < NEG / 2 ? NEG : e;
        }
    }
    const int64_t res = H[W - 1];
    free(H); free(F);
    return res;
}

/* ------------------------------------------------------- one block of a chain */

int orc_block(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n, const orc_scoring *sc,
              const int32_t *top, const int32_t *left, int32_t corner,
              int64_t r0, int64_t c0, int64_t full_m, int64_t full_n, int tie,
              int32_t *bottom, int32_t *right, orc_end *best, uint64_t *bestkey) {
    if (m <= 0 || n <= 0 || r0 < 0 || c0 < 0 || r0 + m > full_m || c0 + n > full_n) return -2;
    orc_geom g;
    if (orc_geometry(full_m, full_n, &g) != 0) tie = ORC_TIE_ROWMAJOR;
    const int32_t ext = sc->gap_extend, open = sc->gap_open;
    int32_t *H = malloc(sizeof(int32_t) * (size_t)n), *F = malloc(sizeof(int32_t) * (size_t)n);
    if (!H || !F) { free(H); free(F); return -3; }
    for (int64_t c = 0; c < n; ++c) {
        H[c] = top ? top[2 * c] : 0;
        F[c] = top ? top[2 * c + 1] : 0;
    }
    int32_t bs = 0;
    uint64_t bk = ~0ULL;
    int64_t br = 0, bc = 0;
    int32_t hd_row = corner;                      /* H[r-1][c0-1] for the current row */
    for (int64_t r = 0; r < m; ++r) {
        int32_t hl = left ? left[2 * r] : 0, el = left ? left[2 * r + 1] : 0;
        int32_t hd = hd_row;
        hd_row = hl;
        const uint8_t ar = a[r];
        for (int64_t c = 0; c < n; ++c) {
            const int32_t f = imax(F[c] + ext, H[c] + open);
            const int32_t e = imax(el + ext, hl + open);
            const int32_t s = (ar == b[c]) ? sc->match : sc->mismatch;
            const int32_t h = imax(imax(0, e), imax(f, hd + s));
            hd = H[c];
            H[c] = h;
            F[c] = f;
            hl = h;
            el = e;
            if (h >= bs && h > 0) {
                const uint64_t key = orc_tie_key(&g, tie, r0 + r, c0 + c);
                if (h > bs || key < bk) { bs = h; bk = key; br = r0 + r; bc = c0 + c; }
            }
        }
        if (right) { right[2 * r] = hl; right[2 * r + 1] = el; }
    }
    if (bottom)
        for (int64_t c = 0; c < n; ++c) { bottom[2 * c] = H[c]; bottom[2 * c + 1] = F[c]; }
    best->score = bs;
    best->row = bs > 0 ? br : 0;
    best->col = bs > 0 ? bc : 0;
    *bestkey = bs > 0 ? bk : ~0ULL;
    free(H); free(F);
    return 0;
}
