/*
 * refemu_cuda.h -- a host-only stand-in for the few CUDA runtime / device
 * facilities that the reference SWalign sources use, so that its own kernel
 * and host files (src/FindAlignment.cuh, src/TraceBack.cuh, src/SWkernel.cuh,
 * src/SWutils.cpp, src/Crosspointer.cpp, src/Builders.cpp, src/FASTA.cpp)
 * compile unchanged with g++ and run on the CPU.
 *
 * TEST INFRASTRUCTURE ONLY: this is part of the oracle's reference build.  It is
 * never linked into the product library.
 *
 * Model:
 *   - device memory is host memory (cudaMalloc = calloc with slack bytes so that
 *     the reference's small over-reads past an allocation read zeros instead of
 *     faulting, like a device allocation rounded up to its granularity);
 *   - a kernel launch runs the blocks of the grid one after another, and the
 *     threads of one block as real host threads that meet at a spinning barrier
 *     for __syncthreads();  the reference's blocks never exchange data inside one
 *     launch, so running them in sequence is faithful;
 *   - threadIdx / blockIdx are thread_local, blockDim / gridDim are globals set
 *     by the launcher;
 *   - texture<char> + tex1Dfetch read the bound linear buffer (0 outside it).
 */
#ifndef REFEMU_CUDA_H_
#define REFEMU_CUDA_H_

#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define __global__
#define __device__
#define __host__
#define __shared__

struct int2 { int x, y; };
struct int3 { int x, y, z; };
struct char4 { signed char x, y, z, w; };
struct dim3 { unsigned int x, y, z; };

static inline int2 make_int2(int x, int y) { int2 r; r.x = x; r.y = y; return r; }

static inline int max(int a, int b) { return a > b ? a : b; }
static inline int min(int a, int b) { return a < b ? a : b; }

extern thread_local dim3 threadIdx;
extern thread_local dim3 blockIdx;
extern dim3 blockDim;
extern dim3 gridDim;

void __syncthreads(void);

template <class T> struct texture {
    const T *ptr;
    size_t bytes;
};
template <class T> static inline T tex1Dfetch(const texture<T> &t, int i) {
    if (t.ptr == NULL || i < 0 || (size_t)i * sizeof(T) >= t.bytes) return (T)0;
    return t.ptr[i];
}

typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorInvalidValue = 1, cudaErrorMemoryAllocation = 2,
       cudaErrorInvalidConfiguration = 9 };
enum cudaMemcpyKind { cudaMemcpyHostToHost = 0, cudaMemcpyHostToDevice = 1,
                      cudaMemcpyDeviceToHost = 2, cudaMemcpyDeviceToDevice = 3 };
enum cudaFuncCache { cudaFuncCachePreferNone = 0, cudaFuncCachePreferShared = 1 };

typedef struct refemu_event *cudaEvent_t;

struct cudaDeviceProp {
    char name[256];
    int major, minor;
    int multiProcessorCount;
    int maxThreadsDim[3];
    size_t totalGlobalMem;
};

cudaError_t cudaMalloc(void **p, size_t size);
cudaError_t cudaFree(void *p);
cudaError_t cudaMemset(void *p, int v, size_t size);
cudaError_t cudaMemcpy(void *dst, const void *src, size_t size, cudaMemcpyKind kind);
cudaError_t cudaDeviceSynchronize(void);
cudaError_t cudaGetDeviceCount(int *n);
cudaError_t cudaGetDeviceProperties(cudaDeviceProp *p, int dev);
cudaError_t cudaSetDevice(int dev);
const char *cudaGetErrorString(cudaError_t e);
cudaError_t cudaEventCreate(cudaEvent_t *e);
cudaError_t cudaEventDestroy(cudaEvent_t e);
cudaError_t cudaEventRecord(cudaEvent_t e, int stream);
cudaError_t cudaEventSynchronize(cudaEvent_t e);
cudaError_t cudaEventElapsedTime(float *ms, cudaEvent_t a, cudaEvent_t b);
template <class F> static inline cudaError_t cudaFuncSetCacheConfig(F, cudaFuncCache) { return cudaSuccess; }
template <class T> static inline cudaError_t cudaBindTexture(size_t *off, texture<T> &t, const void *p, size_t bytes) {
    if (off) *off = 0;
    t.ptr = (const T *)p;
    t.bytes = bytes;
    return cudaSuccess;
}
template <class T> static inline cudaError_t cudaUnbindTexture(texture<T> &t) {
    t.ptr = NULL;
    t.bytes = 0;
    return cudaSuccess;
}

#endif
