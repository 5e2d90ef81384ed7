/*
 * swb200.h -- C ABI of the B200-native Smith-Waterman / Gotoh local-alignment
 * library (libswb200.so), a drop-in for the alignment path of SWalign
 * (Sterbic/Projekt-2012).
 *
 * Conventions shared by every entry point
 *   - Plain C types, caller-owned inputs, no CUDA or C++ types in signatures.
 *   - Every call returns an int status (SWB_OK = 0 or a SWB_E* code) and never
 *     exits the process; swb_last_error() gives a one-line reason.
 *   - Orientation is the reference's: the longer sequence is the "rows"
 *     sequence (the reference's `first` after the swap in src/SWutils.cpp:83-88;
 *     equal lengths keep argument order), the shorter one the "cols" sequence.
 *     Coordinates are 0-based (row in rows sequence, col in cols sequence); the
 *     CLI prints the end cell 1-based like src/main.cu:224.
 *   - Scores are exact int32.  Bytes are compared as they are (any byte value).
 *   - One context per host thread; a context owns one CUDA device and its
 *     buffers, which it reuses from call to call.
 */
#ifndef SWB200_H_
#define SWB200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define SWB_OK            0
#define SWB_EINVAL        1  /* bad argument (the reference exits -1 for these)   */
#define SWB_ENOMEM        2  /* host or device allocation failed                  */
#define SWB_ENOMEM_BUDGET 3  /* request does not fit the context's HBM budget     */
#define SWB_ETIMEOUT      4  /* a bounded device wait ran out                      */
#define SWB_ECUDA         5  /* CUDA runtime error (the reference exits -2)        */
#define SWB_EUNSUPPORTED  6  /* size or option outside what this library supports */
#define SWB_EBUSY         7  /* queue full / request slot unavailable              */
#define SWB_ENOTFOUND     8  /* unknown request id                                 */

/* ---------------------------------------------------------------- types */

/* Replaces `scoring` (src/SWutils.h:15-20; `first` = gap_open).  A gap of
 * length L costs gap_open + (L-1)*gap_extend (src/FindAlignment.cuh:54-56). */
typedef struct {
    int32_t match;
    int32_t mismatch;
    int32_t gap_open;
    int32_t gap_extend;
} swb_scoring;

/* Replaces `TracebackScore` (src/SWutils.h:34-39): a cell where the alignment
 * crosses a special row.  gap = 1 when the path crosses that row inside a
 * vertical gap; score is the forward value of the path's state at that cell. */
typedef struct {
    int32_t gap;
    int32_t score;
    int64_t row;
    int64_t col;
} swb_xpoint;

/* Tie rule among cells that share the best score. */
#define SWB_TIE_REFERENCE 0u   /* the shipped reference's thread-ownership order  */
#define SWB_TIE_ROWMAJOR  1u   /* first cell in row-major order                   */

/* Flags for swb_align_pair / swb_align_pair_device. */
#define SWB_FLAG_TIE_ROWMAJOR  0x1u  /* default is SWB_TIE_REFERENCE              */
#define SWB_FLAG_SCORE_ONLY    0x2u  /* score and end cell only (stage 1)          */
#define SWB_FLAG_NO_SPECIAL    0x4u  /* stage 1 without special-row checkpoints    */
/* Test hook of swb_align_pair[_device]: strip 0 never hands its bottom row to
 * strip 1, so strip 1's first wait runs out after wait_limit_ms and the call
 * returns SWB_ETIMEOUT with the context still usable.  Pairs of one strip (at
 * most 448 rows) have no wait and are unaffected. */
#define SWB_FLAG_TEST_WITHHOLD 0x80000000u
/* Test hook of swb_batch_align[_device]: the packed 16-bit scoring pass takes
 * every pair, also those whose best score may not fit 16 bits; a pair that
 * reaches the limit is detected and scored again in int32, so results do not
 * change.  Without it only pairs whose score is bounded below the limit are
 * packed. */
#define SWB_FLAG_TEST_PACK_ANY 0x40000000u

typedef struct {
    int32_t score;
    int64_t end_row, end_col;       /* 0-based; (0,0) when the best score is 0      */
    int64_t start_row, start_col;   /* first aligned cell; = end when score-only    */
    int32_t swapped;                /* 1: argument A was shorter and became cols    */
    int64_t rows, cols;             /* lengths in the rows / cols orientation       */
    double  stage1_ms;              /* device time of the scoring wavefront         */
    double  stage2_ms;              /* device + host time of traceback              */
    double  total_ms;               /* wall time of the call                        */
    /* alignment, library-owned until swb_result_free(): ops[i] in {'M','I','D'}
     * from start to end.  'M' aligns rows[r] with cols[c]; 'I' is cols[c]
     * against a gap; 'D' is rows[r] against a gap. */
    int64_t n_ops;
    char   *ops;
    /* crosspoints in the reference's output order (src/main.cu:245-248):
     * [start (score 0), one per special row of height xpoint_interval crossed,
     *  end (best score)]; library-owned until swb_result_free(). */
    int64_t     n_xpoints;
    swb_xpoint *xpoints;
    int32_t     xpoint_interval;    /* rows between reference special rows (4*T)    */
    int32_t     special_interval;   /* rows between this run's HBM special rows     */
    int64_t     special_bytes;      /* HBM held by special rows for this call       */
    int32_t     kernel_launches;    /* this library's kernels launched by the call  */
    int64_t     host_bytes;         /* of special_bytes, kept in pinned host memory */
} swb_result;

typedef struct {
    int32_t  device;                /* CUDA device ordinal                           */
    uint64_t hbm_budget_bytes;      /* cap on special rows/columns; 0 = 64 GiB      */
    int32_t  special_interval;      /* special-row spacing in rows; 0 = autotune    */
    int32_t  verbose;               /* bit 0: progress lines on stderr; bit 1: record
                                       the stage-1 strip trace (swb_trace_copy)     */
    uint64_t cuda_stream;           /* a cudaStream_t of the caller to run on, cast
                                       to an integer; 0 = the context's own stream */
    uint32_t wait_limit_ms;         /* bound of every wait of one strip for the strip
                                       above on the GPU; past it the launch stops
                                       and the call returns SWB_ETIMEOUT (the
                                       reference exits -2 on any CUDA error,
                                       src/SWutils.cpp:19-24); 0 = 20,000 ms      */
    uint64_t host_spill_bytes;      /* pinned host memory the special rows or columns
                                       of one call may use beyond hbm_budget_bytes
                                       (the reference appends its special rows to
                                       disk files, src/Builders.cpp:41-61); the
                                       kernels write them through a mapped pointer
                                       and the traceback reads its blocks back;
                                       0 = none (over the budget: level-1 grid)  */
} swb_options;

typedef struct swb_ctx swb_ctx;

/* ---------------------------------------------------------------- calls */

void swb_options_default(swb_options *opts);

/* Creates a context on opts->device (opts may be NULL for defaults). */
int swb_ctx_create(const swb_options *opts, swb_ctx **out);
void swb_ctx_destroy(swb_ctx *ctx);

/* Last error message of the context (or of the thread when ctx is NULL). */
const char *swb_last_error(const swb_ctx *ctx);

/* Replaces initScoringValues (src/SWutils.cpp:26-47): parses with atoi and
 * rejects match < 1 or mismatch/gap_open/gap_extend > -1 with SWB_EINVAL. */
int swb_scoring_parse(const char *match, const char *mismatch, const char *gap_open,
                      const char *gap_extend, swb_scoring *out);

/* Replaces the reference's stage-1 dk loop (src/main.cu:161-214) and its
 * stage 2 (src/Crosspointer.cpp:104-338, driven through kernelWrapperTB,
 * src/main.cu:17-100): aligns host sequences a (length la) and b (length lb).
 * The longer one becomes rows.  Result buffers are library-owned; release them
 * with swb_result_free(). */
int swb_align_pair(swb_ctx *ctx, const uint8_t *a, int64_t la, const uint8_t *b, int64_t lb,
                   const swb_scoring *sc, uint32_t flags, swb_result *out);

/* Same as swb_align_pair but with the sequences already in device memory of the
 * context's device (d_rows is the longer sequence, d_cols the shorter one;
 * rows >= cols is required). */
int swb_align_pair_device(swb_ctx *ctx, const void *d_rows, int64_t rows, const void *d_cols,
                          int64_t cols, const swb_scoring *sc, uint32_t flags, swb_result *out);

void swb_result_free(swb_result *res);

/* Reference launch shape and padding for lengths (rows >= cols):
 * src/SWutils.cpp:233-253 and src/FASTA.cpp:107-134.  Returns SWB_EUNSUPPORTED
 * when the reference could not launch (cols < 4). */
int swb_reference_geometry(int64_t rows, int64_t cols, int32_t *G, int32_t *T, int64_t *P1,
                           int64_t *P2);

/* Copies special row `idx` of the context's last call (row (idx+1)*interval - 1)
 * as (H, F) int32 pairs into host memory out[2*cols]; *interval receives the
 * spacing.  The reference keeps these rows in temp/row_<R> files
 * (src/Builders.cpp:41-61, read back at src/Crosspointer.cpp:94-102). */
int swb_special_row_copy(swb_ctx *ctx, int64_t idx, int32_t *out, int64_t cols, int64_t *interval);

/* One block of a pair split into blocks: the step of the multi-GPU column-chunk
 * chain (swb200/chain.py), where GPU g owns a range of columns, walks it in
 * blocks of rows and passes its right border to GPU g+1.  The reference runs
 * one pair on one GPU (src/main.cu:125-126) and has no counterpart; this is the
 * row recurrence of src/FindAlignment.cuh:54-56 over a sub-rectangle whose
 * boundaries come from its neighbours instead of the zeroed buffers of
 * src/SWutils.cpp:144-168.
 *   block    rows [row_origin, +rows) x cols [col_origin, +cols) of a full_rows x
 *            full_cols matrix (rows = the longer sequence); d_rows / d_cols are
 *            the block's own bytes (device memory)
 *   d_top    (H, F) int32 pairs of row row_origin - 1 over the block's columns,
 *            or NULL at the matrix's top edge (zeros)
 *   d_left   (H, E) int32 pairs of column col_origin - 1 over the block's rows,
 *            or NULL at the left edge (zeros); corner = H[row_origin-1][col_origin-1]
 *   d_bottom receives (H, F) of the block's last row (cols pairs), or NULL; needs
 *            rows to be a multiple of 512
 *   d_right  receives (H, E) of the block's last column (rows pairs), or NULL
 * The best cell comes back in whole-matrix coordinates with its tie key: over
 * all blocks the highest score, then the smallest key, is the pair's result
 * (row, col = -1 and key = ~0 when no cell of the block is positive).  flags:
 * SWB_FLAG_TIE_ROWMAJOR.  Runs on the context's stream and returns when the
 * outputs are written. */
typedef struct {
    int32_t  score;
    int64_t  row, col;
    uint64_t key;
    double   stage1_ms;
} swb_block_best;
int swb_score_block_device(swb_ctx *ctx, const void *d_rows, int64_t rows, const void *d_cols, int64_t cols,
                           const int32_t *d_top, const int32_t *d_left, int32_t corner, int64_t row_origin,
                           int64_t col_origin, int64_t full_rows, int64_t full_cols, const swb_scoring *sc,
                           uint32_t flags, int32_t *d_bottom, int32_t *d_right, swb_block_best *out);

/* Score and end cell of one pair, for callers that cannot allocate device
 * memory.  No counterpart in the reference (its stage 1 allocates its buffers
 * with cudaMalloc, src/SWutils.cpp:144-168).  Callers inside another framework's
 * memory pool, under a no-allocation policy, or that must not fail on device
 * memory pass the sequences (device memory of `device`, rows >= cols) and a host
 * result; the kernel's scratch is a fixed array inside this library (about
 * 16.1 MiB per device that loads it, held until exit).  Limits: cols <=
 * SWB_NOALLOC_MAX_COLS, rows <= SWB_NOALLOC_MAX_ROWS, else SWB_EUNSUPPORTED.
 * The call cannot be captured into a CUDA graph (it copies its result to the
 * host and waits): on a stream that is capturing it returns SWB_EINVAL and
 * leaves the capture intact.  The first call on a device looks up the array's
 * device address.  That first call also loads the array's module, which
 * commits its memory and can fail with SWB_ECUDA (out of memory): callers that must
 * not fail later make it at start-up, where a call with rows = cols = 0 does only
 * this set-up.  The address is kept for the process: after a cudaDeviceReset of
 * the device it is stale, so do not call this entry point on a device that was
 * reset.  Calls on one device that overlap on the GPU race on the shared array.  `cuda_stream` is a cudaStream_t cast to an integer
 * (0 = legacy default stream); the call returns after the result is on the host.
 * Score-only (no traceback).  Error text: swb_noalloc_last_error(). */
#define SWB_NOALLOC_MAX_COLS (1 << 20)
#define SWB_NOALLOC_MAX_ROWS (1 << 25)
typedef struct {
    int32_t score;
    int64_t end_row, end_col;
} swb_score;
int swb_score_pair_noalloc(int32_t device, const void *d_rows, int64_t rows, const void *d_cols,
                           int64_t cols, const swb_scoring *sc, uint32_t flags, uint64_t cuda_stream,
                           swb_score *out);
const char *swb_noalloc_last_error(void);

/* ---------------------------------------------------------------- batches
 *
 * Many independent pairs of uneven length in one persistent launch.  No
 * counterpart in the reference, which aligns one pair per process run
 * (src/main.cu:102-249); each pair gets exactly the result swb_align_pair()
 * gives it alone (score, end cell, tie rule, alignment and crosspoints). */

/* One pair of a batch: byte ranges of the batch's sequence buffer. */
typedef struct {
    int64_t a_off, a_len;
    int64_t b_off, b_len;
} swb_pair_ref;

typedef struct {
    int32_t score;
    int32_t swapped;                /* 1: A was shorter and became cols             */
    int64_t end_row, end_col;       /* 0-based, rows = longer sequence              */
    int64_t start_row, start_col;   /* traced pairs; = end otherwise                */
    int64_t ops_off, n_ops;         /* traced pairs: ops[ops_off, +n_ops) of the result */
    int64_t xp_off, n_xpoints;      /* traced pairs: xpoints[xp_off, +n_xpoints)    */
    int32_t traced;                 /* 1: alignment and crosspoints were computed   */
    int32_t xpoint_interval;        /* reference special-row spacing of this pair   */
} swb_batch_item;

typedef struct {
    int64_t npairs;
    swb_batch_item *items;          /* in the order of the pairs argument           */
    char *ops;                      /* 'M'/'I'/'D' of every traced pair             */
    int64_t ops_bytes;
    swb_xpoint *xpoints;            /* [start, crosspoints, end] of every traced pair */
    int64_t n_xpoints;
    int64_t n_traced;
    int64_t cells;                  /* sum of rows * cols                           */
    double stage1_ms;               /* device time of the batched scoring launch    */
    double stage2_ms;               /* device + host time of the traced pairs       */
    double total_ms;                /* wall time of the call                        */
    int32_t kernel_launches;
} swb_batch_result;

/* Aligns npairs pairs whose sequences are byte ranges of the host buffer seq
 * (seq_bytes long).  Scores and end cells of every pair; the alignment and
 * crosspoints of the ceil(trace_frac * npairs) best-scoring pairs (ties: lower
 * index first; trace_frac in [0, 1]).  flags: SWB_FLAG_TIE_ROWMAJOR.  Result
 * buffers are library-owned until swb_batch_result_free(). */
int swb_batch_align(swb_ctx *ctx, const uint8_t *seq, int64_t seq_bytes, const swb_pair_ref *pairs,
                    int64_t npairs, const swb_scoring *sc, uint32_t flags, double trace_frac,
                    swb_batch_result *out);
/* Same with the sequence buffer already in device memory of the context's device. */
int swb_batch_align_device(swb_ctx *ctx, const void *d_seq, int64_t seq_bytes, const swb_pair_ref *pairs,
                           int64_t npairs, const swb_scoring *sc, uint32_t flags, double trace_frac,
                           swb_batch_result *out);
void swb_batch_result_free(swb_batch_result *res);

/* ---------------------------------------------------------------- serving
 *
 * A request loop with continuous batching.  No counterpart in the reference
 * (one pair per process, src/main.cu:102-249).  Requests are admitted against
 * an HBM budget for their sequences and special rows/columns.  Short requests
 * run in iterations: each iteration batches every admitted short request into
 * one scoring launch plus one batched traceback, and requests that arrive during
 * an iteration join the next one.  Long requests (rows * cols above long_cells)
 * run one at a time in a second lane on their own stream.  Their scoring grid
 * leaves reserve_sms SMs for the short iterations, so both lanes' work overlaps
 * on the device.  A request's result (score, end and start cells, alignment,
 * crosspoints) is exactly what swb_align_pair() returns for the same pair. */

typedef struct swb_server swb_server;

typedef struct {
    int32_t  device;
    uint64_t hbm_budget_bytes;  /* admission budget (sequences + special rows/columns); 0 = 64 GiB */
    int64_t  long_cells;        /* rows * cols above which a request runs in the long lane; 0 = 2^32 */
    int32_t  max_batch;         /* most short requests per iteration; 0 = 8192                   */
    int32_t  reserve_sms;       /* SMs kept for short iterations while a long request runs; 0 = 4  */
    uint32_t flags;             /* SWB_FLAG_TIE_ROWMAJOR                                          */
} swb_server_options;

typedef struct {
    double  queued_ms;          /* submit -> admission                                         */
    double  run_ms;             /* admission -> result                                         */
    double  total_ms;           /* submit -> result                                            */
    int32_t lane;               /* 0 short (batched iterations), 1 long                        */
    int32_t batch_size;         /* requests in the iteration that ran it (1 in the long lane)  */
} swb_request_info;

typedef struct {
    int64_t submitted, completed, failed;
    int64_t iterations;         /* short-lane iterations                                       */
    int64_t max_batch_seen;     /* largest short iteration                                     */
    int64_t long_completed;
    uint64_t peak_reserved_bytes; /* largest admitted footprint at one time                   */
    int64_t cells_completed;
} swb_server_stats;

void swb_server_options_default(swb_server_options *o);
int swb_server_create(const swb_server_options *o, const swb_scoring *sc, swb_server **out);
/* Copies the two sequences and queues the request; *id identifies it.  A request
 * whose footprint exceeds the whole budget fails with SWB_ENOMEM_BUDGET here. */
int swb_server_submit(swb_server *s, const uint8_t *a, int64_t la, const uint8_t *b, int64_t lb, uint64_t *id);
/* Waits up to timeout_ms (< 0: forever) for request id.  SWB_OK: *out holds the
 * result (release with swb_result_free()) and the request is forgotten;
 * SWB_ETIMEOUT: not finished yet; SWB_ENOTFOUND: unknown id; any other code:
 * the request failed (swb_server_last_error()) and is forgotten. */
int swb_server_wait(swb_server *s, uint64_t id, int64_t timeout_ms, swb_result *out, swb_request_info *info);
int swb_server_stats_get(swb_server *s, swb_server_stats *st);
const char *swb_server_last_error(swb_server *s);
/* Finishes the requests already admitted, drops queued ones, stops the lanes. */
void swb_server_destroy(swb_server *s);

/* Stage-1 strip trace of the context's last call when options.verbose has bit 1
 * set: per strip {start ns, end ns, SM id} from %globaltimer / %smid, written to
 * out[3*strips] (cap entries available); *count receives the strip count. */
int swb_trace_copy(swb_ctx *ctx, int64_t *out, int64_t cap, int64_t *count);

/* ------------------------------------------------------------ gap lists
 * The alignment of a result as the gap lists the reference's renderer reads
 * (visualOutput, src/Visualisation.cpp:11-127; it was never called there): per
 * sequence, records {begin, length} meaning `length` gap characters stand
 * before the base at 0-based index `begin` of that sequence.  "first" is the
 * rows sequence of the result (the longer one, A unless swapped), "second" the
 * columns sequence.  Runs of 'I' open gaps in the first sequence, runs of 'D'
 * in the second. */
typedef struct swb_gap {
    int32_t begin;
    int32_t length;
} swb_gap;

/* Writes up to *_cap records to first / second (either may be NULL with cap 0)
 * and the full record counts to *n_first / *n_second.  SWB_EINVAL when result
 * or a count pointer is NULL, when the operation string is malformed, or when a
 * buffer is too small (the counts are still written). */
int swb_gap_lists(const swb_result *result, swb_gap *first, int64_t first_cap, int64_t *n_first,
                  swb_gap *second, int64_t second_cap, int64_t *n_second);

/* The same lists as the reference's binary gap-list files: consecutive native
 * int32 pairs (begin, length), the layout visualOutput reads with fread. */
int swb_gap_lists_write(const swb_result *result, const char *first_path, const char *second_path);

/* ---------------------------------------------------------------- FASTA
 * Reads a FASTA file.  flags = 0: the reference loader's rules exactly
 * (FASTAsequence::load, src/FASTA.cpp:39-86): one record; the first byte must be
 * '>'; the name is the first line without '>' and its last character (at most
 * 199 bytes read); the first 299 bytes of that line are skipped; every other
 * byte except '
' and '
' is sequence, unchanged.  With SWB_FASTA_MULTI every
 * line starting with '>' opens a record whose name is that whole line (any
 * length, without '>' and the line end), lines starting with ';' are comments,
 * and blanks, tabs and line ends are dropped from sequences.  SWB_FASTA_UPPER
 * folds a-z to A-Z in sequences (the kernels compare bytes as they are).
 * *records receives `*count` records owned by the caller (swb_fasta_free).
 * SWB_EINVAL for a missing file or one that does not start with '>'. */
#define SWB_FASTA_MULTI 0x1u
#define SWB_FASTA_UPPER 0x2u

typedef struct swb_fasta_record {
    char *name;     /* NUL-terminated */
    uint8_t *seq;
    int64_t len;
} swb_fasta_record;

int swb_fasta_load(const char *path, uint32_t flags, swb_fasta_record **records, int64_t *count);
void swb_fasta_free(swb_fasta_record *records, int64_t count);

/* Library version string. */
const char *swb_version(void);

#ifdef __cplusplus
}
#endif
#endif
