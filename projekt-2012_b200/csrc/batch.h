// batch.h -- internal declarations of the batched wavefront (batch.cu), used by
// the batched entry points (batch_host.cpp) and the serving loop (serve.cpp).
#pragma once

#include <cstdint>

#include "swb_internal.h"

namespace swb {

// One pair of a batch on the device.  Rows are the longer sequence (m >= n >= 1).
struct BatchPair {
    int64_t row_off, col_off;  // byte offsets of rows / cols in the batch's sequence buffer
    int64_t hbuf_off;          // first hbuf entry of the pair (n entries; pairs with one strip use none)
    int64_t sr_off, sc_off;    // first special-row / special-column entry (store pass only)
    int32_t m, n;
    int32_t unit0;             // work unit u of this launch runs strip u - unit0 of the pair
    int32_t nstrips;           // strips of the whole pair
    int32_t slot;              // index of the pair's record in gbest / pbest
    int32_t sc_every;          // store pass: a special column every sc_every columns (power of two)
    int32_t sr_every;          // store pass: a special row every sr_every strips
    int32_t ufirst, ucount;    // this launch's units of the pair: [ufirst, ufirst + ucount)
    int32_t pad_;
    TieGeom tie;               // tie rule of the pair (reference launch shape of its lengths)
    // boundary pass only (a sub-rectangle of a larger matrix): (H, F) of the row
    // above and (H, E) of the column to the left (nullptr: matrix edge, zero);
    // the corner H is top[-1] when both exist
    const int2 *top, *left;
};

// What a launch computes besides the best cells.
enum BatchMode : int32_t {
    kBatchScore = 0,       // scores only
    kBatchStores = 1,      // special rows / columns of every pair
    kBatchBounds = 2,      // special rows / columns of sub-rectangles with top / left boundaries
};

// Uniform arguments of one batched launch.
struct BatchArgs {
    const uint8_t *seq;        // sequence bytes of the rows (CMP mode)
    const uint8_t *cseq;       // sequence bytes of the columns (CMP mode; usually seq)
    const uint8_t *rcode;      // TAB mode: per-byte code of seq
    const uint32_t *ctab;      // TAB mode: per-byte table word of cseq
    int32_t open, ext, gx, mt1, mm1;
    uint32_t tab_hi;
    const BatchPair *pairs;
    const int32_t *unit_pair;  // work unit -> index into pairs; units are claimed in this order
    const int32_t *unit_strip; // if set, work unit -> strip of its pair; else the strip is u - unit0
    int64_t nunits;
    const int64_t *nunits_dev; // if set, the unit count is read here (graphed launches) instead
    int4 *hbuf;
    int32_t *gbest;            // per pair slot: best H seen so far
    BestRec *ubest;            // per strip: best cell, at ufirst + strip of its pair
    int32_t *ctl;              // [0] unit counter, [1] error code, [2] abort flag
    int2 *srows, *scols;       // store pass: special rows (H, F) / columns (H, E) of every pair
    int64_t wait_limit;        // bound of each wait for the strip above, in SM clock cycles; 0 = default
};

// Two pairs scored side by side in packed 16-bit lanes (batch16.cu): half 0 is
// pair a (low 16 bits of every lane register), half 1 pair b.  Both have the
// same strip count; the packed rectangle is M = max(m) rows x N = max(n) columns.
struct PackedPair {
    int64_t row_off[2], col_off[2];  // byte offsets of each pair's rows / cols in the sequence buffer
    int64_t hbuf_off;                // first of the N hand-off entries (packs of more than one strip)
    int32_t m[2], n[2];              // m = n = 0: an empty half
    int32_t M, N;
    int32_t unit0, nstrips;          // strip s keeps its two best records at ubest[2 (unit0 + s) + half]
    int32_t whole, pad_;             // 1: one work item, one warp runs every strip in turn;
                                     // 0: one work item per strip, chained across warps
    int32_t slot[2];                 // pbest / gbest / saturation slot of each half
    TieGeom tie[2];
};

// Uniform arguments of one packed launch (TAB mode only: table words and row codes).
struct Batch16Args {
    const uint8_t *rcode;
    const uint32_t *ctab;
    uint32_t open2, ext2, gx2;  // gap_open, gap_extend, max of both in both halves
    int32_t open;
    uint32_t mm4;               // the table word of a column past a pair's end (a mismatch for every code)
    int32_t sat_lim;            // a half's column maximum (H + open) at or above this flags its pair
    const PackedPair *pairs;
    const int2 *items;          // work item -> (packed pair, strip); claimed in this order
    int64_t nunits;             // work items
    int4 *hbuf;
    int32_t *gbest;             // per slot: best H seen so far
    BestRec *ubest;             // per strip of every packed pair: two records (half 0, half 1)
    int32_t *ctl;               // [0] unit counter, [1] error code, [2] abort flag
    int32_t *sat;               // per slot: 1 when the pair reached the 16-bit limit
    int64_t wait_limit;
};

// Rows per lane of the packed kernel: 14 (448-row strips) unless the batch
// autotuner picks 8 (256-row strips, less padding below short pairs).
constexpr int kBatch16R = 14;
constexpr int kBatch16RShort = 8;

cudaError_t batch16_configure();
// Warps of a full packed launch (the grid batch16_launch uses at most).
int batch16_resident_warps(int R, int sms, int max_blocks);
// R: kBatch16R or kBatch16RShort; the packed pairs' strip counts must use it.
cudaError_t batch16_launch(const Batch16Args &a, int R, int sms, int max_blocks, int64_t npacked, BestRec *pbest,
                           cudaStream_t st);

// Rows per lane of the batched kernel's store passes (their strips are 512 rows,
// the walker's block height); score-only passes may use 8 (256-row strips).
constexpr int kBatchR = 16;
constexpr int kBatchStripRows = 32 * kBatchR;

// One call of a graphed batch.  The captured kernels take the address of this
// header, which never moves, and the host rewrites the header before every
// replay, so one graph serves every call with the same grid; only the two
// scoring kernels also take the launch's BatchArgs as a parameter, set on the
// instantiated graph per replay.
struct GraphHdr {
    BatchArgs ba;             // the scoring launch (descriptors, units, work buffers)
    BestRec *pbest;           // per entry of ba.pairs (slot k)
    int64_t npairs;           // entries of ba.pairs
    int64_t nunits;           // work units of the scoring launch (ba.nunits_dev points here)
    int64_t seq_bytes;        // bytes at ba.seq
    int64_t hbuf_entries;     // hand-off entries to reset
    void *walk_args;          // traced graphs: walker arguments per pair (traceback.cu's layout)
    int64_t *walk_states;     // traced graphs: walker state per pair
    uint32_t *walk_dir;       // traced graphs: walker direction scratch (8 CTAs per SM)
    uint8_t *lut;             // byte -> code (written by the decide kernel)
    uint32_t *presence;       // 256-bit byte bitmap (all zero between calls)
    int32_t *out;             // [0..3] the launch's control words, [4] the decided mode
    uint32_t x1;              // table word: match ^ mismatch byte
    int32_t tab_ok;           // the scoring values fit the table words
    int32_t tab;              // 1: at most four distinct byte values (set on the device)
    int32_t pad_;
};

// Queues the graphed batch's kernels on st (normally under stream capture):
// reset and alphabet scan, mode decision, encode, the scoring kernel of either
// mode (the other one returns at once), the per-pair merge.  With traced = true
// the scoring kernel keeps every pair's special rows and columns.  Grids are
// sized for calls of at most max_units work units (and pairs).  ev_mid, if
// non-null, is recorded (as an external event) after the merge.
cudaError_t batch_graph_enqueue(const GraphHdr *d_hdr, bool traced, int R, int sms, int max_blocks,
                                int64_t max_units, cudaEvent_t ev_mid, cudaStream_t st);
// The two scoring kernels of such a graph (table path, compare path): their
// parameters (BatchArgs, header address) are set on the instantiated graph
// before every replay.
void batch_graph_scoring_funcs(bool traced, int R, const void **f);

// Launches the batched wavefront over units [0, a.nunits) (a.ctl must be zeroed
// first), then merges the strips' best cells of pairs [0, npairs) of a.pairs
// into pbest[slot] (which holds the pair's best so far, or an invalid record).
// Every strip a launch runs must have its predecessor strip either earlier in the
// same launch's unit order or finished by an earlier launch.  `mode` selects
// what is stored.  max_blocks > 0 caps the grid (the rest of the GPU stays free
// for other work).
cudaError_t batch_launch(const BatchArgs &a, bool tab, BatchMode mode, int R, int sms, int max_blocks,
                         int64_t npairs, BestRec *pbest, cudaStream_t st);
// Byte presence flags over a buffer (TAB-mode choice) and the TAB encodings of
// every byte of seq (rcode[i] = lut[seq[i]], ctab[i] = table word of seq[i]).
cudaError_t batch_encode(const uint8_t *seq, int64_t bytes, const uint8_t *d_lut, uint8_t *rcode, uint32_t *ctab,
                         int32_t mt1, int32_t mm1, uint32_t *tab_hi, cudaStream_t st);
int batch_max_blocks_per_sm(bool tab, BatchMode mode);
// Warps of a full batched launch of that mode (the grid batch_launch uses at most).
int batch_resident_warps(bool tab, BatchMode mode, int sms, int max_blocks);
// Rows per lane of score-only batched launches (16 unless SWB_BATCH_R overrides).
int batch_score_rows_per_lane();

// Host batch with every pair traced, in one scoring pass that keeps the stores
// (the serving loop's iteration).  Same contract as swb_batch_align(..., 1.0, ...).
int batch_align_all_traced(swb_ctx *c, const uint8_t *h_seq, int64_t seq_bytes, const swb_pair_ref *pairs,
                           int64_t npairs, const swb_scoring *sc, uint32_t flags, swb_batch_result *out);

}  // namespace swb
