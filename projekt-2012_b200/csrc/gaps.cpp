// gaps.cpp -- an alignment as the reference's gap lists (swb_gap_lists*).  The
// reference's renderer visualOutput (src/Visualisation.cpp:11-127) reads, per
// sequence, binary records {int begin, int length}: `length` gap characters
// before the base at index `begin`; the reference never produced those files.
// Derived here from the result's operation string: a run of 'I' (a column base
// against a gap) is a gap in the first (rows) sequence before its next base, a
// run of 'D' a gap in the second (columns) sequence.
#include <cstdio>
#include <vector>

#include "ctx.h"

namespace {

int derive(const swb_result *r, std::vector<swb_gap> &first, std::vector<swb_gap> &second) {
    if (!r || (r->n_ops > 0 && !r->ops)) return SWB_EINVAL;
    int64_t ri = r->start_row, ci = r->start_col;
    int64_t i = 0;
    while (i < r->n_ops) {
        const char op = r->ops[i];
        int64_t j = i;
        while (j < r->n_ops && r->ops[j] == op) ++j;
        const int64_t run = j - i;
        if (op == 'M') {
            ri += run;
            ci += run;
        } else if (op == 'I') {
            if (ri > INT32_MAX || run > INT32_MAX) return SWB_EUNSUPPORTED;
            first.push_back(swb_gap{(int32_t)ri, (int32_t)run});
            ci += run;
        } else if (op == 'D') {
            if (ci > INT32_MAX || run > INT32_MAX) return SWB_EUNSUPPORTED;
            second.push_back(swb_gap{(int32_t)ci, (int32_t)run});
            ri += run;
        } else {
            return SWB_EINVAL;
        }
        i = j;
    }
    return SWB_OK;
}

}  // namespace

extern "C" int swb_gap_lists(const swb_result *result, swb_gap *first, int64_t first_cap, int64_t *n_first,
                             swb_gap *second, int64_t second_cap, int64_t *n_second) {
    if (!result || !n_first || !n_second || first_cap < 0 || second_cap < 0 || (first_cap > 0 && !first) ||
        (second_cap > 0 && !second))
        return swb::ctx_fail(nullptr, SWB_EINVAL, "swb_gap_lists: bad arguments");
    std::vector<swb_gap> a, b;
    const int rc = derive(result, a, b);
    if (rc != SWB_OK) return swb::ctx_fail(nullptr, rc, "swb_gap_lists: malformed or oversized alignment");
    *n_first = (int64_t)a.size();
    *n_second = (int64_t)b.size();
    for (size_t k = 0; k < a.size() && (int64_t)k < first_cap; ++k) first[k] = a[k];
    for (size_t k = 0; k < b.size() && (int64_t)k < second_cap; ++k) second[k] = b[k];
    if ((int64_t)a.size() > first_cap || (int64_t)b.size() > second_cap)
        return swb::ctx_fail(nullptr, SWB_EINVAL, "swb_gap_lists: buffer too small");
    return SWB_OK;
}

extern "C" int swb_gap_lists_write(const swb_result *result, const char *first_path, const char *second_path) {
    if (!result || !first_path || !second_path)
        return swb::ctx_fail(nullptr, SWB_EINVAL, "swb_gap_lists_write: bad arguments");
    std::vector<swb_gap> a, b;
    const int rc = derive(result, a, b);
    if (rc != SWB_OK) return swb::ctx_fail(nullptr, rc, "swb_gap_lists_write: malformed or oversized alignment");
    const std::vector<swb_gap> *lists[2] = {&a, &b};
    const char *paths[2] = {first_path, second_path};
    for (int k = 0; k < 2; ++k) {
        FILE *f = std::fopen(paths[k], "wb");
        if (!f) return swb::ctx_fail(nullptr, SWB_EINVAL, "cannot open %s for writing", paths[k]);
        for (const swb_gap &g : *lists[k]) {
            const int32_t rec[2] = {g.begin, g.length};
            if (std::fwrite(rec, sizeof rec, 1, f) != 1) {
                std::fclose(f);
                return swb::ctx_fail(nullptr, SWB_EINVAL, "cannot write %s", paths[k]);
            }
        }
        if (std::fclose(f) != 0) return swb::ctx_fail(nullptr, SWB_EINVAL, "cannot write %s", paths[k]);
    }
    return SWB_OK;
}
