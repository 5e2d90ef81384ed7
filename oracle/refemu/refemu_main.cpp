/*
 * refemu_main.cpp -- CPU build of the reference SWalign (Sterbic/Projekt-2012).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the driver of the oracle's reference
 * build: it compiles the reference's own kernel headers (src/FindAlignment.cuh,
 * src/TraceBack.cuh, src/SWkernel.cuh) and links its own host files
 * (src/SWutils.cpp, src/Crosspointer.cpp, src/Builders.cpp, src/FASTA.cpp),
 * taken from where they lie in the reference checkout, against the host stand-in
 * of the CUDA runtime in shim/refemu_cuda.h.  Nothing of the reference is copied
 * here: this file supplies only (1) the stand-in runtime, (2) the kernel
 * launcher that runs CUDA threads as host threads, (3) the extern "C"
 * kernelWrapperTB that the reference's Crosspointer.cpp calls (its body in the
 * reference is src/main.cu:17-100, which g++ cannot parse because of the <<< >>>
 * launch syntax), and (4) a main() that performs the same sequence of calls as
 * the reference's src/main.cu:102-249.
 *
 * Usage: swalign_emu <seqA.fasta> <seqB.fasta> <match> <mismatch> <open> <ext>
 *                    [--stage1-only]
 * Machine-readable results go to stderr as
 *   "REFEMU score <s> <row1> <col1>"      (1-based, as printed by main.cu:224)
 *   "REFEMU geom <G> <T> <P1> <P2>"
 *   "REFEMU xpoint <i> <row> <col> <score> <gap>"   (0-based, main.cu:245-248)
 * The reference's own stdout chatter is left as it is.
 */
#include <atomic>
#include <chrono>
#include <functional>
#include <thread>
#include <vector>

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include "refemu_cuda.h"

#include "Defines.h"
#include "FASTA.h"
#include "SWutils.h"
#include "Builders.h"
#include "FindAlignment.cuh"
#include "TraceBack.cuh"
#include "Crosspointer.h"

/* ---------------------------------------------------------------- threads */

thread_local dim3 threadIdx;
thread_local dim3 blockIdx;
dim3 blockDim;
dim3 gridDim;

/* The reference kernels declare `extern __shared__ int2 iHbuffer[]`; blocks run
 * one after another here, so one array stands for every block's shared memory. */
int2 iHbuffer[4096];

static std::atomic<int> g_bar_count{0};
static std::atomic<int> g_bar_gen{0};
static int g_bar_n = 1;

void __syncthreads(void) {
    int gen = g_bar_gen.load(std::memory_order_acquire);
    if (g_bar_count.fetch_add(1, std::memory_order_acq_rel) + 1 == g_bar_n) {
        g_bar_count.store(0, std::memory_order_relaxed);
        g_bar_gen.fetch_add(1, std::memory_order_acq_rel);
    } else {
        unsigned spins = 0;
        while (g_bar_gen.load(std::memory_order_acquire) == gen)
            if (++spins > 256) std::this_thread::yield();
    }
}

/* A pool of host threads, one per CUDA thread of a block. */
struct BlockPool {
    std::vector<std::thread> workers;
    std::atomic<long> go{0};
    std::atomic<int> done{0};
    std::atomic<bool> quit{false};
    std::function<void()> task;
    unsigned block = 0;

    explicit BlockPool(int n) {
        for (int i = 0; i < n; ++i)
            workers.emplace_back([this, i] { loop(i); });
    }
    ~BlockPool() {
        quit.store(true);
        go.fetch_add(1);
        for (auto &w : workers) w.join();
    }
    void loop(int idx) {
        long seen = 0;
        for (;;) {
            unsigned spins = 0;
            while (go.load(std::memory_order_acquire) == seen)
                if (++spins > 256) std::this_thread::yield();
            seen = go.load(std::memory_order_acquire);
            if (quit.load()) return;
            threadIdx.x = idx; threadIdx.y = 0; threadIdx.z = 0;
            blockIdx.x = block; blockIdx.y = 0; blockIdx.z = 0;
            task();
            done.fetch_add(1, std::memory_order_acq_rel);
        }
    }
    void run_block(unsigned b, const std::function<void()> &f) {
        task = f;
        block = b;
        done.store(0);
        go.fetch_add(1, std::memory_order_acq_rel);
        unsigned spins = 0;
        while (done.load(std::memory_order_acquire) != (int)workers.size())
            if (++spins > 256) std::this_thread::yield();
    }
};

static BlockPool *g_pool = NULL;

/* Runs one grid: blocks in sequence, the threads of a block concurrently. */
static void launch(int blocks, int threads, const std::function<void()> &kernel) {
    if (blocks <= 0 || threads <= 0) {
        printf("Error in line %d\n", __LINE__);
        exitWithMsg("invalid configuration argument", -2);
    }
    if (g_pool == NULL || (int)g_pool->workers.size() != threads) {
        delete g_pool;
        g_pool = new BlockPool(threads);
    }
    gridDim.x = blocks; gridDim.y = gridDim.z = 1;
    blockDim.x = threads; blockDim.y = blockDim.z = 1;
    g_bar_n = threads;
    g_bar_count.store(0);
    for (int b = 0; b < blocks; ++b) g_pool->run_block(b, kernel);
}

/* ---------------------------------------------------------------- runtime */

static const size_t kSlack = 4096;

cudaError_t cudaMalloc(void **p, size_t size) {
    *p = calloc(1, size + kSlack);
    return *p ? cudaSuccess : cudaErrorMemoryAllocation;
}
cudaError_t cudaFree(void *p) { free(p); return cudaSuccess; }
cudaError_t cudaMemset(void *p, int v, size_t size) { memset(p, v, size); return cudaSuccess; }
cudaError_t cudaMemcpy(void *dst, const void *src, size_t size, cudaMemcpyKind) {
    memmove(dst, src, size);
    return cudaSuccess;
}
cudaError_t cudaDeviceSynchronize(void) { return cudaSuccess; }
cudaError_t cudaGetDeviceCount(int *n) { *n = 1; return cudaSuccess; }
cudaError_t cudaGetDeviceProperties(cudaDeviceProp *p, int) {
    memset(p, 0, sizeof(*p));
    strcpy(p->name, "host emulation of a compute-capability 3.5 device");
    p->major = 3; p->minor = 5;               /* a generation the reference accepts */
    p->multiProcessorCount = 13;
    p->maxThreadsDim[0] = 1024; p->maxThreadsDim[1] = 1024; p->maxThreadsDim[2] = 64;
    p->totalGlobalMem = (size_t)6 << 30;
    return cudaSuccess;
}
cudaError_t cudaSetDevice(int) { return cudaSuccess; }
const char *cudaGetErrorString(cudaError_t e) { return e == cudaSuccess ? "no error" : "emulated CUDA error"; }

struct refemu_event { std::chrono::steady_clock::time_point t; };
cudaError_t cudaEventCreate(cudaEvent_t *e) { *e = new refemu_event(); return cudaSuccess; }
cudaError_t cudaEventDestroy(cudaEvent_t e) { delete e; return cudaSuccess; }
cudaError_t cudaEventRecord(cudaEvent_t e, int) { e->t = std::chrono::steady_clock::now(); return cudaSuccess; }
cudaError_t cudaEventSynchronize(cudaEvent_t) { return cudaSuccess; }
cudaError_t cudaEventElapsedTime(float *ms, cudaEvent_t a, cudaEvent_t b) {
    *ms = std::chrono::duration<float, std::milli>(b->t - a->t).count();
    return cudaSuccess;
}

/* ------------------------------------------------- stage-2 kernel wrapper */

/* Same dispatch as the reference's extern "C" wrapper (src/main.cu:17-100):
 * kernel codes from src/Defines.h:11-13, launch shape from the Crosspointer. */
extern "C" void kernelWrapperTB(Crosspointer *xp, int dk, TracebackScore *devLast, int kernel) {
    LaunchConfig lc = xp->getStdLaunchConfig();
    HorizontalBuffer hb = xp->getHBuffer();
    VerticalBuffer vb = xp->getVBuffer();
    char *row = xp->getDevRow();
    char *col = xp->getDevColumn();
    int h = xp->getSrHeight();
    scoring v = xp->getValues();
    bool gap = xp->getGap();
    int target = xp->getTarget().score;
    int off = xp->getInitVBusOffset();
    int2 *vbo = xp->getDevVBusOut();
    if (kernel == TRACEBACK_LAST_SHORT) {
        launch(lc.blocks, lc.threads, [&] { tracebackLastShort(dk, hb, vb, row, h, col, h, v, gap, devLast, target, off); });
    } else if (kernel == TRACEBACK_LAST_LONG) {
        launch(lc.blocks, lc.threads, [&] { tracebackLastLong(dk, hb, vb, row, h, col, h, v, gap, devLast, target, off); });
    } else if (kernel == TRACEBACK_SHORT_LONG) {
        launch(lc.blocks, lc.threads, [&] { tracebackShort(dk, hb, vb, row, h, col, h, v, vbo, gap, off); });
        launch(lc.blocks, lc.threads, [&] { tracebackLong(dk, hb, vb, row, h, col, h, v, vbo, gap, off); });
    } else {
        exitWithMsg("Unknown kernel type passed to wrapper.", -1);
    }
}

/* ------------------------------------------------------------------ main */

int main(int argc, char *argv[]) {
    if (argc != 7 && argc != 8) {
        printf("Expected 6 input arguments, not %d!\n\n", argc - 1);
        return -1;
    }
    bool stage1_only = (argc == 8 && strcmp(argv[7], "--stage1-only") == 0);

    /* The reference keeps its special rows in append-only files temp/row_<R>
     * under the working directory; give every run a fresh one. */
    char *fa = realpath(argv[1], NULL);
    char *fb = realpath(argv[2], NULL);
    if (!fa || !fb) exitWithMsg("An error has occured while loading input sequences.", -1);
    char work[] = "/tmp/refemu_XXXXXX";
    if (!mkdtemp(work) || chdir(work) != 0 || mkdir("temp", 0700) != 0)
        exitWithMsg("cannot create a scratch directory", -3);

    FASTAsequence first(fa);
    FASTAsequence second(fb);
    if (!first.load() || !second.load())
        exitWithMsg("An error has occured while loading input sequences.", -1);

    CUDAcard gpu = findBestDevice();
    LaunchConfig config = getLaunchConfig(min(first.getLength(), second.getLength()), gpu);
    SWquery query(&first, &second);
    query.prepare(config);
    scoring values = initScoringValues(argv[3], argv[4], argv[5], argv[6]);

    int scoreSize = sizeof(alignmentScore) * config.blocks * config.threads;
    alignmentScore *score = (alignmentScore *)malloc(scoreSize);
    alignmentScore *devScore = (alignmentScore *)cudaGetSpaceAndSet(scoreSize, 0);
    GlobalBuffer buffer;
    initGlobalBuffer(&buffer, query.getSecond()->getPaddedLength(), config);
    int P1 = query.getFirst()->getPaddedLength();
    int P2 = query.getSecond()->getPaddedLength();
    int D = config.blocks + (int)ceil(((double)P1) / (ALPHA * config.threads)) - 1;
    cudaBindTexture(NULL, texSecond, query.getDevSecond(), P2);
    RowBuilder rowBuilder(P1, P2, &config);
    char *devFirst = query.getDevFirst();

    for (int dk = 0; dk < D + config.blocks; ++dk) {
        launch(config.blocks, config.threads, [&] { shortPhase(dk, buffer.hBuffer, buffer.vBuffer, devFirst, P1, P2, values, devScore); });
        rowBuilder.dumpShort(buffer.hBuffer.up, dk);
        launch(config.blocks, config.threads, [&] { longPhase(dk, buffer.hBuffer, buffer.vBuffer, devFirst, P1, P2, values, devScore); });
        rowBuilder.dumpLong(buffer.hBuffer.up, dk);
    }
    cudaMemcpy(score, devScore, scoreSize, cudaMemcpyDeviceToHost);
    alignmentScore best = getMaxScore(score, config.blocks * config.threads);

    printf("\t>Alignment score: %d at [%d, %d]\n\n", best.score, best.row + 1, best.column + 1);
    fprintf(stderr, "REFEMU geom %d %d %d %d\n", config.blocks, config.threads, P1, P2);
    fprintf(stderr, "REFEMU score %d %d %d\n", best.score, best.row + 1, best.column + 1);
    fflush(stderr);

    cudaUnbindTexture(texSecond);
    cudaFree(devScore);
    freeGlobalBuffer(&buffer);
    free(score);

    if (!stage1_only) {
        Crosspointer xPointer(&query, &gpu, &values, best, rowBuilder.getRowHeight());
        std::vector<TracebackScore> xPoints = xPointer.findCrosspoints();
        printf("Found %d crosspoints:\n", (int)xPoints.size());
        for (size_t i = 0; i < xPoints.size(); ++i) {
            printf("\t>xPoint[%d]: [%d, %d] = %d\n", (int)i, xPoints[i].row, xPoints[i].column, xPoints[i].score);
            fprintf(stderr, "REFEMU xpoint %d %d %d %d %d\n", (int)i, xPoints[i].row, xPoints[i].column,
                    xPoints[i].score, (int)xPoints[i].gap);
        }
        fflush(stderr);
    }

    /* drop the scratch directory */
    char cmd[128];
    snprintf(cmd, sizeof cmd, "rm -rf '%s'", work);
    if (chdir("/") == 0) { int rc = system(cmd); (void)rc; }
    delete g_pool;
    g_pool = NULL;
    free(fa);
    free(fb);
    return 0;
}
