/*
 * swb200_probe.h -- measurement entry points of libswb200.so (not part of the
 * reference-facing ABI; the reference has no counterpart).
 */
#ifndef SWB200_PROBE_H_
#define SWB200_PROBE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Peak cell-update rate of the stage-1 per-cell instruction mix on `device`:
 * every resident thread runs 8 independent cell chains with the same DPX/INT32
 * operations the wavefront issues per cell, with no memory traffic, shuffles or
 * control flow.  Writes cells/s (the int32 cell-update roofline) and the
 * per-op rates of IADD, __viaddmax_s32 and __vimax3_s32 measured alone, in
 * operations per second.  Returns 0 on success. */
int swb_probe_cell_peak(int32_t device, double *cells_per_s, double *iadd_per_s, double *viaddmax_per_s,
                        double *vimax3_per_s, double *elapsed_ms);

/* Dependent-chain latency (SM cycles per operation, one thread) of up to six
 * operations: IADD, max(x + a, b) written in C, __viaddmax_s32, __vimax3_s32,
 * __viaddmax_s32_relu, max(x, b) written in C.  Returns 0 on success. */
int swb_probe_latency(int32_t device, double *cycles_per_op, int32_t nops);

#ifdef __cplusplus
}
#endif
#endif
