// cli.cpp -- the SWalign command line, a drop-in for the reference binary
// (usage README.md:55-63, driver src/main.cu:102-249).
//
//   SWalign <seqA.fasta> <seqB.fasta> <match> <mismatch> <gap_open> <gap_extend>
//
// Kept byte-identical with the reference: the argument-count message and exit
// code (main.cu:107-110), the load and scoring error blocks and exit -1
// (SWutils.cpp:13-17, :36-37), CUDA errors exit -2 (SWutils.cpp:19-24), and the
// result lines
//   "\t>Cell updates per second: %lf GCUPS\n"                 (main.cu:223)
//   "\t>Alignment score: %d at [%d, %d]\n\n"  1-based end     (main.cu:224)
//   "Found %d crosspoints:\n" "\t>xPoint[%d]: [%d, %d] = %d\n" (main.cu:245-248)
// followed by the alignment in the 3-line, 50-column blocks of the reference's
// (never called) visualOutput (src/Visualisation.cpp:62-127); with SWB_GAP_LISTS
// set, also the gap-list files that renderer reads (:11-43).
// Other lines are informational, as in the reference.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "swb200.h"

// A loaded sequence (a view of a swb_fasta_record).
struct Seq {
    std::string name;
    struct Bytes {
        const unsigned char *p;
        size_t n;
        const unsigned char *data() const { return p; }
        size_t size() const { return n; }
    } seq;
    Seq(const char *nm, const unsigned char *p, size_t n) : name(nm), seq{p, n} {}
};

static void exit_with_msg(const char *msg, int code) {
    std::printf("ERROR\n");
    std::printf("%s\n\n", msg);
    std::exit(code);
}

static void render_alignment(const swb_result &r, const unsigned char *rows, const unsigned char *cols) {
    const int kLine = 50;  // PRINT_ROW_LENGTH, src/Visualisation.h:6
    std::printf("\n\tVisual representation of the alignment:\n\n");
    int64_t ri = r.start_row, ci = r.start_col;
    std::string l0, l1, l2;
    for (int64_t i = 0; i < r.n_ops; ++i) {
        const char op = r.ops[i];
        char a = '-', b = '-';
        if (op == 'M') {
            a = (char)rows[ri++];
            b = (char)cols[ci++];
        } else if (op == 'D') {
            a = (char)rows[ri++];
        } else {
            b = (char)cols[ci++];
        }
        l0.push_back(a);
        l2.push_back(b);
        l1.push_back(a == b ? '|' : ' ');
        if ((int)l0.size() == kLine || i + 1 == r.n_ops) {
            std::printf("\t\t%s\n\t\t%s\n\t\t%s\n\n", l0.c_str(), l1.c_str(), l2.c_str());
            l0.clear();
            l1.clear();
            l2.clear();
        }
    }
}

int main(int argc, char *argv[]) {
    std::printf("### Welcome to SWalign (B200 build, %s)\n\n", swb_version());
    const auto t_app = std::chrono::steady_clock::now();
    if (argc != 7) {
        std::printf("Expected 6 input arguments, not %d!\n\n", argc - 1);
        return -1;
    }
    // the reference loader's rules (flags 0): one record, bytes kept as they are
    swb_fasta_record *fa = nullptr, *fb = nullptr;
    int64_t na = 0, nb = 0;
    std::printf("> Loading input sequences... ");
    if (swb_fasta_load(argv[1], 0, &fa, &na) != SWB_OK || swb_fasta_load(argv[2], 0, &fb, &nb) != SWB_OK)
        exit_with_msg("An error has occured while loading input sequences.", -1);
    const Seq A{fa[0].name, fa[0].seq, (size_t)fa[0].len}, B{fb[0].name, fb[0].seq, (size_t)fb[0].len};
    std::printf("DONE\n\n");
    std::printf("First sequence of length %d:\n%s\n\n", (int)A.seq.size(), A.name.c_str());
    std::printf("Second sequence of length %d:\n%s\n\n", (int)B.seq.size(), B.name.c_str());

    swb_options opts;
    swb_options_default(&opts);
    if (const char *d = std::getenv("SWB_DEVICE")) opts.device = std::atoi(d);
    if (const char *b = std::getenv("SWB_HBM_BUDGET_GB")) opts.hbm_budget_bytes = (uint64_t)(std::atof(b) * (1ULL << 30));
    std::printf("> Looking for CUDA capable cards... ");
    swb_ctx *ctx = nullptr;
    if (swb_ctx_create(&opts, &ctx) != SWB_OK) {
        std::printf("Error in line %d\n", __LINE__);
        exit_with_msg(swb_last_error(nullptr), -2);
    }
    std::printf("DONE\n\n");

    swb_scoring sc;
    std::printf("> Initializing scoring values... ");
    if (swb_scoring_parse(argv[3], argv[4], argv[5], argv[6], &sc) != SWB_OK)
        exit_with_msg("One or more scoring values were not usable!", -1);
    std::printf("DONE\n\nScoring values:\n");
    std::printf("\t>Match: %d\n", sc.match);
    std::printf("\t>Mismatch: %d\n", sc.mismatch);
    std::printf("\t>First gap: %d\n", sc.gap_open);
    std::printf("\t>Gap extension: %d\n\n", sc.gap_extend);

    std::printf("> Starting alignment process... ");
    uint32_t flags = 0;
    if (const char *t = std::getenv("SWB_TIE"); t && std::strcmp(t, "rowmajor") == 0) flags |= SWB_FLAG_TIE_ROWMAJOR;
    if (std::getenv("SWB_SCORE_ONLY")) flags |= SWB_FLAG_SCORE_ONLY;
    swb_result res;
    const int rc = swb_align_pair(ctx, A.seq.data(), (int64_t)A.seq.size(), B.seq.data(), (int64_t)B.seq.size(), &sc,
                                  flags, &res);
    if (rc == SWB_EINVAL) exit_with_msg(swb_last_error(ctx), -1);
    if (rc != SWB_OK) {
        std::printf("Error in line %d\n", __LINE__);
        exit_with_msg(swb_last_error(ctx), -2);
    }
    const double app_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_app).count();
    std::printf("DONE\n\n");
    const double gcups = (double)A.seq.size() / 1e6 * (double)B.seq.size() / app_ms;
    std::printf("\t>Kernel executed in %f s\n", res.stage1_ms / 1000.0);
    std::printf("\t>Application executed in %f s\n", app_ms / 1000.0);
    std::printf("\t>Cell updates per second: %lf GCUPS\n", gcups);
    std::printf("\t>Alignment score: %d at [%d, %d]\n\n", res.score, (int)res.end_row + 1, (int)res.end_col + 1);

    if (!(flags & SWB_FLAG_SCORE_ONLY)) {
        std::printf("Found %d crosspoints:\n", (int)res.n_xpoints);
        for (int64_t i = 0; i < res.n_xpoints; ++i)
            std::printf("\t>xPoint[%d]: [%d, %d] = %d\n", (int)i, (int)res.xpoints[i].row, (int)res.xpoints[i].col,
                        res.xpoints[i].score);
        if (res.n_ops > 0) {
            const unsigned char *rows = res.swapped ? B.seq.data() : A.seq.data();
            const unsigned char *cols = res.swapped ? A.seq.data() : B.seq.data();
            render_alignment(res, rows, cols);
            // the reference renderer's binary gap lists, when asked for (SWB_GAP_LISTS=<prefix>
            // writes <prefix>.first.bin and <prefix>.second.bin)
            if (const char *g = std::getenv("SWB_GAP_LISTS")) {
                const std::string p(g);
                if (swb_gap_lists_write(&res, (p + ".first.bin").c_str(), (p + ".second.bin").c_str()) != SWB_OK)
                    std::printf("Gap lists not written: %s\n", swb_last_error(nullptr));
            }
        }
    }
    swb_result_free(&res);
    swb_ctx_destroy(ctx);
    swb_fasta_free(fa, na);
    swb_fasta_free(fb, nb);
    return 0;
}
