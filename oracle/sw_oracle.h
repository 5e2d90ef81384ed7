/*
 * sw_oracle.h -- CPU restatement of the reference SWalign (Sterbic/Projekt-2012)
 * Smith-Waterman / Gotoh local-alignment path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load this library, and only as the checker or the timed
 * CPU baseline.  The product library never links, loads or calls it.
 *
 * Orientation follows the reference: "rows" is the longer sequence (the
 * reference's "first" after the swap in src/SWutils.cpp:83-88; equal lengths
 * keep argument order), "cols" is the shorter one.  All coordinates are 0-based.
 */
#ifndef SW_ORACLE_H_
#define SW_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {            /* src/SWutils.h:15-20 (`first` is the gap-open penalty) */
    int32_t match, mismatch, gap_open, gap_extend;
} orc_scoring;

typedef struct {            /* launch shape + padding of the shipped reference */
    int32_t G, T;           /* blocks, threads: src/SWutils.cpp:233-253          */
    int64_t P1, P2, C;      /* padded rows / cols, column chunk P2/G: FASTA.cpp:107-134 */
} orc_geom;

typedef struct {
    int32_t score;
    int64_t row, col;       /* end cell, 0-based; (0,0) when every cell is 0      */
} orc_end;

enum { ORC_TEXTBOOK = 0,    /* zero boundaries: the H matrix of textbook Gotoh SW */
       ORC_SHIPPED_CARRY = 1 /* the shipped kernels' left boundary carry (see .c)  */ };
enum { ORC_TIE_REFERENCE = 0, /* the shipped kernels' thread-ownership order      */
       ORC_TIE_ROWMAJOR = 1,
       ORC_TIE_BOTH = 2 };    /* orc_stage1_simd only: out[0] reference, out[1] row-major */

/* Returns 0, or -1 when the reference cannot launch (shorter length < 4). */
int orc_geometry(int64_t rows, int64_t cols, orc_geom *g);

/* Ordering key of cell (r, c) under the tie rule (smaller wins among equal H). */
uint64_t orc_tie_key(const orc_geom *g, int tie, int64_t r, int64_t c);

/* Stage 1: best local score and its end cell.  a = rows, b = cols (|a| >= |b|). */
int orc_stage1(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
               const orc_scoring *sc, int semantics, int tie, orc_end *out);

/* Stage 1 on all `threads` host threads (blocked wavefront), textbook semantics.
 * Same result as orc_stage1(..., ORC_TEXTBOOK, tie, ...); also accepts m < n
 * (bands of rows used as timing samples).  Returns elapsed ns in
 * *ns_out when it is not NULL. */
int orc_stage1_mt(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
                  const orc_scoring *sc, int tie, int threads, orc_end *out, int64_t *ns_out);

/* The same result as orc_stage1_mt() from an AVX-512 anti-diagonal wavefront
 * (sw_oracle_simd.c): strips of 16 rows, one row per vector lane.  With tie =
 * ORC_TIE_BOTH, out points to two results (reference order, row-major) found in
 * one pass.  Returns -4 when the CPU has no AVX-512 (callers then use
 * orc_stage1_mt). */
int orc_stage1_simd(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
                    const orc_scoring *sc, int tie, int threads, orc_end *out, int64_t *ns_out);

/* Full H/E/F rows for checking special rows: writes H and F of every row r with
 * (r + 1) % k == 0 into hf[(r + 1) / k - 1][c] as (H, F) pairs (textbook).
 * Returns the number of rows written. */
int64_t orc_special_rows(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
                         const orc_scoring *sc, int64_t k, int32_t *hf, int64_t max_rows);

/* Canonical traceback from end cell (er, ec), textbook semantics, full matrix in
 * memory (m * n bytes).  Precedence: in H, diagonal > E (gap in rows' sequence,
 * horizontal) > F (vertical); in E or F, extend > open.  Writes the operations
 * from start to end into ops ('M' diagonal, 'I' horizontal = column base against
 * a gap, 'D' vertical = row base against a gap), returns their count, and the
 * start cell (first 'M') in *sr, *sc_.  Returns -1 if cap is too small or the
 * matrix does not fit, -2 on bad input. */
int64_t orc_traceback(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
                      const orc_scoring *sc, int64_t er, int64_t ec,
                      char *ops, int64_t cap, int64_t *sr, int64_t *sc_);

/* The same traceback, also reporting the path's crosspoints: for every row X
 * with (X + 1) % xp_interval == 0 that the path crosses, the last path cell on
 * row X (the cell the backward walk enters from row X + 1) as (X, col, forward
 * value of the path at that cell, gap) where gap = 1 when the vertical gap
 * continues across the row boundary; top to bottom, count in *nxp. */
int64_t orc_traceback_xp(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
                         const orc_scoring *sc, int64_t er, int64_t ec,
                         char *ops, int64_t cap, int64_t *sr, int64_t *sc_,
                         int64_t xp_interval, int64_t *xps, int64_t xp_cap, int64_t *nxp);

/* Score of an alignment given as ops from (sr, sc_) (checks a traceback); a run
 * of L same-direction gap characters costs gap_open + (L-1) * max(gap_open,
 * gap_extend), which is what the recurrence gives. */
int64_t orc_score_ops(const uint8_t *a, const uint8_t *b, const orc_scoring *sc,
                      int64_t sr, int64_t sc_, const char *ops, int64_t nops);

/* Best score of an alignment that starts with the diagonal cell (sr, sc_) and ends
 * at (er, ec) (same gap recurrence, no zero floor); INT64_MIN on bad input.  Used
 * to check that a start cell reported by the reference's own stage 2 begins an
 * optimal alignment. */
int64_t orc_anchored_score(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n,
                           const orc_scoring *sc, int64_t sr, int64_t sc_, int64_t er, int64_t ec);

/* One block of a pair split into blocks (the multi-GPU column-chunk chain):
 * rows [r0, r0+m) x cols [c0, c0+n) of a full_m x full_n matrix (a, b point at
 * the block's own bytes), given top[2n] = (H, F) of row r0-1 over the block's
 * columns and left[2m] = (H, E) of column c0-1 over its rows (NULL: the matrix
 * edge, zeros) and corner = H[r0-1][c0-1].  Writes bottom[2n] = (H, F) of its
 * last row and right[2m] = (H, E) of its last column (either may be NULL), and
 * its best cell in whole-matrix coordinates with its tie key (~0 when no cell
 * is positive), so that the best over all blocks with the smallest key among
 * equal scores is the whole matrix's result.  Returns 0, or -2 / -3. */
int orc_block(const uint8_t *a, int64_t m, const uint8_t *b, int64_t n, const orc_scoring *sc,
              const int32_t *top, const int32_t *left, int32_t corner,
              int64_t r0, int64_t c0, int64_t full_m, int64_t full_n, int tie,
              int32_t *bottom, int32_t *right, orc_end *best, uint64_t *bestkey);

#ifdef __cplusplus
}
#endif
#endif
