// traceback.h -- stage 2 of the pair path (crosspoints + alignment) on the GPU.
#pragma once

#include <string>

#include "swb_internal.h"

namespace swb {
namespace tb {

// Special-row spacing (rows) for a pair under the context's HBM budget.
int64_t choose_special_interval(const swb_options &opts, int64_t m, int64_t n);

// Canonical traceback from the end cell in `out` (score, end_row, end_col set by
// stage 1).  Fills out->ops / out->n_ops / start_* / xpoints.  Returns SWB_OK or
// an SWB_E* code with `err` set.
int traceback(cudaStream_t st, const uint8_t *d_rows, int64_t m, const uint8_t *d_cols, int64_t n,
              const swb_scoring *sc, const int2 *d_srows, int64_t nsr, int64_t sr_interval, swb_result *out,
              const uint8_t *h_rows, const uint8_t *h_cols, std::string &err);

}  // namespace tb
}  // namespace swb
