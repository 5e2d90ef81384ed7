// swb_internal.h -- internal declarations shared by the host and device sources
// of libswb200.so.  Not part of the C ABI (include/swb200.h is).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "../../include/swb200.h"

namespace swb {

// Rows handled by one lane of the stage-1 wavefront.  A warp holds a strip of
// 32 * R rows; special rows are kept at multiples of the strip height.
constexpr int kLanes = 32;

// Per-warp best cell: HO is H + gap_open (the kernel works on H + open so that
// the F chain needs one DPX op per row), key orders equal scores.
struct BestRec {
    int32_t ho;
    int32_t valid;
    uint64_t key;
    int64_t row;
    int64_t col;
};

enum TieMode : int32_t { kTieReference = 0, kTieRowMajor = 1 };

struct TieGeom {
    int32_t mode;  // TieMode
    int32_t G, T;  // reference launch shape
    int64_t C;     // reference column chunk P2 / G
};

// Device buffers and scalars for one stage-1 launch over a rectangle of the
// matrix: rows [r_origin, r_origin + m) x cols [c_origin, c_origin + n).
struct Stage1Args {
    const uint8_t *rows;   // device, m bytes (the rectangle's rows)
    const uint8_t *cols;   // device, n bytes
    int64_t m, n;
    int32_t open, ext, gx; // gap_open, gap_extend, max(gap_open, gap_extend)
    int32_t mt1, mm1;      // match - open, mismatch - open
    const uint8_t *rcode;  // TAB mode: per-row code (0..3, 7 = matches nothing)
    const uint32_t *ctab;  // TAB mode: per-column word of (s - open) bytes for codes 0..3
    uint32_t tab_hi;       // TAB mode: (mismatch - open) in all four bytes (codes 4..7)
    int4 *hbuf;            // n entries {H + open, tag, F of the next row, tag}; 0xFF-filled per launch
    int2 *srows;           // special rows [nsr][n] of (H, F), or nullptr
    int64_t sr_every;      // a special row every sr_every strips
    int64_t nsr;           // number of special rows
    int2 *scols;           // special columns [nsc][m] of (H, E), or nullptr
    int32_t sc_every;      // a special column every sc_every columns (power of two)
    int64_t nsc;
    const int2 *top;       // (H, F) of the row above the rectangle, n entries, or nullptr (zero)
    const int2 *left;      // (H, E) of the column left of the rectangle, m entries, or nullptr (zero)
    int32_t corner;        // H above-left of the rectangle
    int64_t r_origin, c_origin;  // rectangle origin in the whole matrix (tie key)
    int64_t nstrips;
    BestRec *wbest;        // one per warp of the grid
    BestRec *best;         // final reduced record
    int32_t *err;          // [0] error code, [1] abort flag, [2] best H seen so far (device-wide)
    int32_t *gbest;        // best H seen so far in this matrix (err + 2 for a single pair)
    int64_t *trace;        // optional: per strip {start ns, end ns, SM id} (globaltimer)
    TieGeom tie;
    int64_t wait_limit;    // bound of each wait for the strip above, in SM clock cycles; 0 = kWaitLimitCycles
    int32_t withhold;      // test hook: strip 0 writes no hand-off entries (SWB_FLAG_TEST_WITHHOLD)
    int2 *bottom;          // optional: (H, F) of the last row, n entries (m a multiple of the strip height)
    int2 *right;           // optional: (H, E) of the last column, m entries
};

// Geometry of the reference's launch (src/SWutils.cpp:233-253) and padding
// (src/FASTA.cpp:107-134).  Returns false when the reference could not launch.
bool reference_geometry(int64_t rows, int64_t cols, int32_t *G, int32_t *T, int64_t *P1,
                        int64_t *P2);

// Stage-1 launch plan (chosen by the host for a pair).
struct Stage1Plan {
    bool tab = false;      // PRMT table substitution (column alphabet of <= 4 bytes)
    bool stores = false;   // run the store-mode kernel even without store buffers (autotuner probes)
    int R = 16;            // rows per lane
    int warps_per_block = 4;
    int blocks = 0;
    int64_t strip_rows = 0;
    int64_t nstrips = 0;
};

// Host entry of stage 1: score and end cell, optional special rows.  All
// pointers in `a` are device pointers owned by the caller.  Returns a CUDA
// error (cudaSuccess on success); a bounded-wait timeout is reported through
// a.err and *timed_out.
cudaError_t stage1_launch(Stage1Args &a, const Stage1Plan &plan, cudaStream_t st);
Stage1Plan stage1_plan(int64_t m, int64_t n, int device_sms, int R_hint, bool tab);
int stage1_max_blocks_per_sm(int R, bool tab);
// 256 presence flags of the bytes of seq (device), for choosing TAB mode.
cudaError_t stage1_presence(const uint8_t *seq, int64_t n, uint32_t *flags, cudaStream_t st);
// TAB-mode encodings: rcode[m] and ctab[n] from a device byte->code table.
cudaError_t stage1_encode(const uint8_t *rows, int64_t m, const uint8_t *cols, int64_t n, const uint8_t *d_lut,
                          uint8_t *rcode, uint32_t *ctab, int32_t mt1, int32_t mm1, uint32_t *tab_hi,
                          cudaStream_t st);

uint64_t tie_key_host(const TieGeom &g, int64_t r, int64_t c);

// Shared-memory carveout preference of the library's kernels on the current
// device (stage1.cu, batch.cu, traceback.cu); called when a context is created.
cudaError_t stage1_configure();
cudaError_t batch_configure();

}  // namespace swb
