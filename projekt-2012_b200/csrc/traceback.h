// traceback.h -- stage 2 of the pair path (crosspoints + alignment) on the GPU.
#pragma once

#include <string>

#include "swb_internal.h"

namespace swb {
struct GraphHdr;
namespace tb {

// Special-row / special-column spacing of stage 1 for a pair.  Direct mode keeps
// the walker's grid (br x 256: the strip height by 256 columns); level-1 mode
// keeps a coarser grid that fits the HBM budget and recomputes each level-1 cell
// on the path with 512 x 256 blocks.
struct Plan {
    bool level1 = false;
    int64_t kr = 512;   // special-row spacing (rows): br (direct) or 3584 x 2^k (level 1)
    int64_t kc = 256;   // special-column spacing (columns), power of two >= 256
    int64_t br = 512;   // block rows of the walker's grid: the stage-1 strip height in direct
                        // mode (448 or 512), 512 in level 1
};
// br: the stage-1 strip height the special rows will come from (a multiple of 32
// up to 512); direct mode when its stores fit the budget.
Plan plan_for(const swb_options &opts, int64_t m, int64_t n, int64_t br = 512);
// Where direct-mode special rows and columns go: both in HBM when they fit the
// budget; else one set (rows first) in pinned host memory when it fits the
// spill and the other fits the budget; else both in host memory when they fit
// the spill.  Returns false when none of these fits (level-1 grid instead).
bool spill_placement(uint64_t hbm, uint64_t spill, uint64_t rows_bytes, uint64_t cols_bytes, bool *rows_host,
                     bool *cols_host);
// Level-1 traceback: cells recomputed per corridor round, and device bytes per
// cell (its 512 x 256 stores and row hand-off buffer).
int64_t level1_corridor_cells(const Plan &plan, int sms);
int64_t level1_cell_store_bytes(const Plan &plan);
cudaError_t walker_configure();

// Inputs of one walker launch over a region [rr0, rr1) x [cc0, cc1).
struct WalkInputs {
    const uint8_t *rows, *cols;   // whole sequences (device)
    int64_t m, n;
    swb_scoring sc;
    int32_t score;
    const int2 *srows, *scols;    // the region's 512 x 256 stores
    int64_t rr0, cc0, rr1, cc1;
    const int2 *rtop, *rleft;     // region boundary (nullptr = matrix edge); the corner H is
                                  // rtop[-1] when both exist
    int32_t xp_interval;
    char *ops;
    int64_t ops_cap;
    int64_t *xps;
    int64_t xp_cap;
    int64_t *dstate;              // device copy of the walker state
    int64_t br;                   // block rows of the region's grid (0: 512)
};


size_t walk_args_bytes();
int state_slots();
int slot_r();
int slot_c();
int slot_state();
int slot_nops();
int slot_nxp();
int slot_done();
int slot_err();
int slot_start_r();
int slot_start_c();
int block_rows();
int block_cols();

// Device scratch the orchestration needs (owned by the caller's context).
struct Scratch {
    void *(*ensure)(void *owner, int which, size_t bytes);  // returns device memory or nullptr
    // copies between host and device through the owner's pinned staging on its stream
    cudaError_t (*get)(void *owner, void *dst, const void *dev_src, size_t bytes);
    cudaError_t (*put)(void *owner, void *dev_dst, const void *src, size_t bytes);
    void *owner;
};
enum ScratchSlot {
    kScrOps = 0, kScrXps, kScrState, kScrSrows2, kScrScols2, kScrHbuf, kScrWbest, kScrBest, kScrErr,
    kScrGdir, kScrBlk, kScrMap, kScrWalkErr,
    kScrL1Pairs, kScrL1Units, kScrL1Hbuf, kScrL1Gbest, kScrL1Ubest, kScrL1Pbest, kScrL1Ctl, kScrSlots
};

// Walks the path from host_state's cell through the region of `in` (until the
// start cell or the region's top/left edge): rounds of a predicted corridor of
// whole blocks precomputed in parallel, then walked by one warp.
int walk_region(cudaStream_t st, int sms, const WalkInputs &in, int64_t *host_state, const Scratch &scr,
                std::string &err, int32_t *launches);

// Walks n independent pairs (each region is its pair's whole matrix) with one
// launch; d_args holds n * walk_args_bytes() bytes, d_states n * state_slots()
// int64 (initial states are copied from host_states, final ones back to it),
// d_dir walk_batch_dir_bytes(sms, n) bytes of direction scratch.
int walk_batch(cudaStream_t st, int sms, const WalkInputs *in, int64_t n, void *d_args, int64_t *d_states,
               void *d_dir, int64_t *host_states, const Scratch &scr, std::string &err);
size_t walk_batch_dir_bytes(int sms, int64_t n);

// Graphed batches (the header's walk_args / walk_states / walk_dir hold every
// pair of the batch): writes the walker arguments of n pairs into dst (host
// memory, n * walk_args_bytes() bytes, states at d_states + i * state_slots()),
// and queues the walker's init and walk kernels for calls of at most max_pairs
// pairs, up to walk_graph_ctas(sms) CTAs whose direction scratch is
// walk_batch_dir_bytes(sms, walk_graph_ctas(sms)).
void pack_walk_args(const WalkInputs *in, int64_t n, int64_t *d_states, void *dst);
cudaError_t walk_graph_enqueue(const GraphHdr *d_hdr, int sms, int64_t max_pairs, cudaStream_t st);
int64_t walk_graph_ctas(int sms);

// Canonical traceback from the end cell in `out` (score, end_row, end_col set by
// stage 1), using the stage-1 stores laid out by `plan`.  Fills out->ops,
// out->n_ops, start_*, xpoints.  Returns SWB_OK or an SWB_E* code with `err`.
int traceback(cudaStream_t st, int sms, const uint8_t *d_rows, int64_t m, const uint8_t *d_cols, int64_t n,
              const swb_scoring *sc, const Plan &plan, const int2 *d_srows, const int2 *d_scols, swb_result *out,
              const Scratch &scr, std::string &err, int32_t *launches);

}  // namespace tb
}  // namespace swb
