// traceback.cu -- stage 2 (GPU traceback); filled in by the traceback kernels.
#include "traceback.h"

namespace swb {
namespace tb {

int64_t choose_special_interval(const swb_options &opts, int64_t m, int64_t n) {
    (void)m; (void)n;
    return opts.special_interval > 0 ? opts.special_interval : 0;
}

int traceback(cudaStream_t st, const uint8_t *d_rows, int64_t m, const uint8_t *d_cols, int64_t n,
              const swb_scoring *sc, const int2 *d_srows, int64_t nsr, int64_t sr_interval, swb_result *out,
              const uint8_t *h_rows, const uint8_t *h_cols, std::string &err) {
    (void)st; (void)d_rows; (void)m; (void)d_cols; (void)n; (void)sc; (void)d_srows; (void)nsr;
    (void)sr_interval; (void)out; (void)h_rows; (void)h_cols;
    err = "traceback is not built yet";
    return SWB_EUNSUPPORTED;
}

}  // namespace tb
}  // namespace swb
