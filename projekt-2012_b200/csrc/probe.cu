// probe.cu -- the cell-update roofline: the stage-1 per-cell DPX/INT32 mix run
// at full occupancy with no memory traffic, and the single-op rates.
#include <cstdio>

#include "swb_internal.h"
#include "../../include/swb200_probe.h"

namespace swb {
namespace {

constexpr int kChains = 8;

// One cell of stage1.cu's step() per chain and iteration: compare/select of the
// substitution score, E, t, t + open, HO, F' and half a three-way max.
__global__ void cell_mix_kernel(const int32_t *in, int32_t *out, int iters) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    int32_t HO[kChains], E[kChains], f[kChains], hod[kChains], cm[kChains];
    const int32_t ra = in[0] + (tid & 3), cb0 = in[1], mt1 = in[2], mm1 = in[3];
    const int32_t ext = in[4], open = in[5], gx = in[6];
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
        HO[c] = in[7] + c + tid;
        E[c] = in[8] - c;
        f[c] = in[9] + c;
        hod[c] = in[10] + tid;
        cm[c] = in[11];
    }
    int32_t cb = cb0;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) {
            const int32_t s1 = (ra == cb + c) ? mt1 : mm1;
            const int32_t e = __viaddmax_s32(E[c], ext, HO[c]);
            const int32_t t = __viaddmax_s32_relu(hod[c], s1, e);
            const int32_t to = t + open;
            const int32_t ho = __viaddmax_s32(f[c], open, to);
            f[c] = __viaddmax_s32(f[c], gx, to);
            hod[c] = HO[c];
            cm[c] = __vimax3_s32(cm[c], ho, HO[c]);
            HO[c] = ho;
            E[c] = e;
        }
        cb ^= 1;
    }
    int32_t acc = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc ^= HO[c] ^ E[c] ^ f[c] ^ cm[c] ^ hod[c];
    out[tid] = acc;
}

// op: 0 = IADD, 1 = __viaddmax_s32, 2 = __vimax3_s32; 8 independent chains.
__global__ void single_op_kernel(const int32_t *in, int32_t *out, int iters, int op) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    int32_t x[kChains];
    const int32_t a = in[0] | 1, b = in[1];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = in[2] + c * tid;
    if (op == 0) {
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int c = 0; c < kChains; ++c) x[c] = x[c] + a;
    } else if (op == 1) {
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int c = 0; c < kChains; ++c) x[c] = __viaddmax_s32(x[c], a, b + it);
    } else {
        for (int it = 0; it < iters; ++it)
#pragma unroll
            for (int c = 0; c < kChains; ++c) x[c] = __vimax3_s32(x[c], a + it, b);
    }
    int32_t acc = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc ^= x[c];
    out[tid] = acc;
}

// Dependent-chain latency in SM cycles per operation, one thread.
// op: 0 IADD, 1 max(x + a, b) in plain C, 2 __viaddmax_s32, 3 __vimax3_s32,
//     4 __viaddmax_s32_relu, 5 max(x, b) in plain C
__global__ void latency_kernel(const int32_t *in, int32_t *out, int iters, int op, long long *cycles) {
    int32_t x = in[0];
    const int32_t a = in[1], b = in[2];
    const long long t0 = clock64();
    switch (op) {
        case 0: for (int i = 0; i < iters; ++i) x = x + a; break;
        case 1: for (int i = 0; i < iters; ++i) x = max(x + a, b + i); break;
        case 2: for (int i = 0; i < iters; ++i) x = __viaddmax_s32(x, a, b + i); break;
        case 3: for (int i = 0; i < iters; ++i) x = __vimax3_s32(x, a + i, b); break;
        case 4: for (int i = 0; i < iters; ++i) x = __viaddmax_s32_relu(x, a, b + i); break;
        default: for (int i = 0; i < iters; ++i) x = max(x, b + i); break;
    }
    const long long t1 = clock64();
    out[0] = x;
    *cycles = t1 - t0;
}

}  // namespace
}  // namespace swb

extern "C" int swb_probe_latency(int32_t device, double *cycles_per_op, int32_t nops) {
    using namespace swb;
    if (cudaSetDevice(device) != cudaSuccess) return SWB_ECUDA;
    int32_t hin[4] = {3, -2, -7, 0};
    int32_t *din = nullptr, *dout = nullptr;
    long long *dcyc = nullptr;
    if (cudaMalloc(&din, sizeof hin) != cudaSuccess || cudaMalloc(&dout, 16) != cudaSuccess ||
        cudaMalloc(&dcyc, sizeof(long long)) != cudaSuccess)
        return SWB_ENOMEM;
    cudaMemcpy(din, hin, sizeof hin, cudaMemcpyHostToDevice);
    const int iters = 1 << 16;
    for (int op = 0; op < nops && op < 6; ++op) {
        long long best = -1;
        for (int rep = 0; rep < 3; ++rep) {
            latency_kernel<<<1, 1>>>(din, dout, iters, op, dcyc);
            long long c = 0;
            cudaMemcpy(&c, dcyc, sizeof c, cudaMemcpyDeviceToHost);
            if (best < 0 || c < best) best = c;
        }
        cycles_per_op[op] = (double)best / iters;
    }
    cudaFree(din);
    cudaFree(dout);
    cudaFree(dcyc);
    return cudaGetLastError() == cudaSuccess ? SWB_OK : SWB_ECUDA;
}

extern "C" int swb_probe_cell_peak(int32_t device, double *cells_per_s, double *iadd_per_s,
                                   double *viaddmax_per_s, double *vimax3_per_s, double *elapsed_ms) {
    using namespace swb;
    if (cudaSetDevice(device) != cudaSuccess) return SWB_ECUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int threads = 256;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cell_mix_kernel, threads, 0);
    const int blocks = sms * (per_sm > 0 ? per_sm : 1);
    const int iters = 4096;
    int32_t hin[16] = {65, 67, 6, 2, -2, -5, -2, -5, 0, -3, -5, 0, 0, 0, 0, 0};
    int32_t *din = nullptr, *dout = nullptr;
    if (cudaMalloc(&din, sizeof hin) != cudaSuccess) return SWB_ENOMEM;
    if (cudaMalloc(&dout, sizeof(int32_t) * (size_t)blocks * threads) != cudaSuccess) {
        cudaFree(din);
        return SWB_ENOMEM;
    }
    cudaMemcpy(din, hin, sizeof hin, cudaMemcpyHostToDevice);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float ms = 0.f;
    // warm-up, then the best of three timed launches
    cell_mix_kernel<<<blocks, threads>>>(din, dout, iters / 4);
    float best = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0);
        cell_mix_kernel<<<blocks, threads>>>(din, dout, iters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    const double cells = (double)blocks * threads * iters * kChains;
    if (cells_per_s) *cells_per_s = cells / (best * 1e-3);
    if (elapsed_ms) *elapsed_ms = best;
    double *outs[3] = {iadd_per_s, viaddmax_per_s, vimax3_per_s};
    for (int op = 0; op < 3; ++op) {
        single_op_kernel<<<blocks, threads>>>(din, dout, iters / 4, op);
        float b2 = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            cudaEventRecord(e0);
            single_op_kernel<<<blocks, threads>>>(din, dout, iters * 4, op);
            cudaEventRecord(e1);
            cudaEventSynchronize(e1);
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < b2) b2 = ms;
        }
        if (outs[op]) *outs[op] = (double)blocks * threads * iters * 4 * kChains / (b2 * 1e-3);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(din);
    cudaFree(dout);
    return cudaGetLastError() == cudaSuccess ? SWB_OK : SWB_ECUDA;
}
