/*
 * visual_main.cpp -- CPU build of the reference's alignment renderer.
 *
 * TEST INFRASTRUCTURE ONLY.  Links the reference's own visualOutput
 * (src/Visualisation.cpp:11-129, taken from where it lies in the reference
 * checkout; the reference never calls it) against the host stand-in of the CUDA
 * headers in shim/, and calls it once:
 *
 *   visual_emu <first.bin> <second.bin> <first.gaps> <second.gaps> <sx> <sy> <ex> <ey>
 *
 * first.bin / second.bin hold the two sequences as raw bytes (the rows sequence
 * first, as the reference's "first" after its swap, src/SWutils.cpp:83-88); the
 * gap files are the {int begin, int length} records that swb_gap_lists_write
 * produces; (sx, sy) / (ex, ey) are the first and last aligned cells, 0-based.
 * The renderer's output goes to stdout unchanged.
 *
 * visualOutput dereferences its gap-list iterators without checking for the end
 * (Visualisation.cpp:68,88), so a list that has run out reads past the vector.
 * The caller therefore ends each gap file with one record {-1, 0}, whose begin
 * matches no offset, so the renderer never advances past it.
 */
#include <stdio.h>
#include <stdlib.h>

#include <string>
#include <vector>

#include "refemu_cuda.h"

void visualOutput(char *firstSequence, char *secondSequence, const char *firstFilename,
                  const char *secondFilename, int2 startPoint, int2 endPoint);

static std::vector<char> slurp(const char *path) {
    std::vector<char> v;
    FILE *f = fopen(path, "rb");
    if (!f) {
        fprintf(stderr, "cannot open %s\n", path);
        exit(2);
    }
    char buf[1 << 16];
    size_t k;
    while ((k = fread(buf, 1, sizeof buf, f)) > 0) v.insert(v.end(), buf, buf + k);
    fclose(f);
    v.push_back(0);
    return v;
}

int main(int argc, char *argv[]) {
    if (argc != 9) {
        fprintf(stderr, "usage: visual_emu first.bin second.bin first.gaps second.gaps sx sy ex ey\n");
        return 2;
    }
    std::vector<char> first = slurp(argv[1]), second = slurp(argv[2]);
    int2 start, end;
    start.x = atoi(argv[5]);
    start.y = atoi(argv[6]);
    end.x = atoi(argv[7]);
    end.y = atoi(argv[8]);
    visualOutput(first.data(), second.data(), argv[3], argv[4], start, end);
    fflush(stdout);
    return 0;
}
