// fasta_api.cpp -- swb_fasta_load / swb_fasta_free: the reference loader's rules
// (src/FASTA.cpp:39-86, shared with the CLI through fasta_load) and a multi-record
// reader for inputs the reference loader mishandles (several records, headers
// longer than 299 bytes, comments, lower case).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.h"
#include "fasta.h"

namespace {

struct Rec {
    std::string name;
    std::vector<unsigned char> seq;
};

bool read_all(const char *path, std::vector<unsigned char> &out) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    unsigned char buf[1 << 16];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) out.insert(out.end(), buf, buf + got);
    std::fclose(f);
    return true;
}

bool parse_multi(const std::vector<unsigned char> &d, std::vector<Rec> &recs) {
    if (d.empty() || d[0] != '>') return false;
    size_t i = 0;
    while (i < d.size()) {
        size_t e = i;
        while (e < d.size() && d[e] != '\n') ++e;
        size_t le = e;
        if (le > i && d[le - 1] == '\r') --le;
        if (d[i] == '>') {
            recs.emplace_back();
            recs.back().name.assign(reinterpret_cast<const char *>(d.data()) + i + 1, le - i - 1);
        } else if (d[i] != ';') {
            for (size_t k = i; k < le; ++k) {
                const unsigned char b = d[k];
                if (b == ' ' || b == '\t' || b == '\r') continue;
                recs.back().seq.push_back(b);
            }
        }
        i = e + 1;
    }
    return true;
}

}  // namespace

extern "C" int swb_fasta_load(const char *path, uint32_t flags, swb_fasta_record **records, int64_t *count) {
    if (!path || !records || !count) return swb::ctx_fail(nullptr, SWB_EINVAL, "swb_fasta_load: bad arguments");
    *records = nullptr;
    *count = 0;
    std::vector<Rec> recs;
    if (flags & SWB_FASTA_MULTI) {
        std::vector<unsigned char> d;
        if (!read_all(path, d) || !parse_multi(d, recs))
            return swb::ctx_fail(nullptr, SWB_EINVAL, "%s: not a FASTA file", path);
    } else {
        swb::FastaRecord r;
        if (!swb::fasta_load(path, &r)) return swb::ctx_fail(nullptr, SWB_EINVAL, "%s: not a FASTA file", path);
        recs.push_back(Rec{r.name, std::move(r.seq)});
    }
    if (flags & SWB_FASTA_UPPER)
        for (Rec &r : recs)
            for (unsigned char &b : r.seq)
                if (b >= 'a' && b <= 'z') b = (unsigned char)(b - 'a' + 'A');
    auto *out = (swb_fasta_record *)std::calloc(recs.size() ? recs.size() : 1, sizeof(swb_fasta_record));
    if (!out) return swb::ctx_fail(nullptr, SWB_ENOMEM, "out of host memory");
    for (size_t k = 0; k < recs.size(); ++k) {
        out[k].name = (char *)std::malloc(recs[k].name.size() + 1);
        out[k].seq = (uint8_t *)std::malloc(recs[k].seq.size() ? recs[k].seq.size() : 1);
        if (!out[k].name || !out[k].seq) {
            swb_fasta_free(out, (int64_t)recs.size());
            return swb::ctx_fail(nullptr, SWB_ENOMEM, "out of host memory");
        }
        std::memcpy(out[k].name, recs[k].name.c_str(), recs[k].name.size() + 1);
        if (!recs[k].seq.empty()) std::memcpy(out[k].seq, recs[k].seq.data(), recs[k].seq.size());
        out[k].len = (int64_t)recs[k].seq.size();
    }
    *records = out;
    *count = (int64_t)recs.size();
    return SWB_OK;
}

extern "C" void swb_fasta_free(swb_fasta_record *records, int64_t count) {
    if (!records) return;
    for (int64_t k = 0; k < count; ++k) {
        std::free(records[k].name);
        std::free(records[k].seq);
    }
    std::free(records);
}
