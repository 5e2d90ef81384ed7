// fasta.cpp -- see fasta.h.  Follows src/FASTA.cpp:39-86: the header is read with
// a 200-byte fgets for the name and a 300-byte fgets to skip it, so a header
// longer than 299 bytes spills into the sequence exactly as in the reference.
#include "fasta.h"

#include <cstdio>
#include <cstring>

namespace swb {

bool fasta_load(const char *path, FastaRecord *out) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return false;
    char c[301];
    std::memset(c, 0, sizeof c);
    if (!std::fgets(c, 200, f) || c[0] != '>') {
        std::fclose(f);
        return false;
    }
    const size_t len = std::strlen(c);
    out->name.assign(len >= 2 ? c + 1 : c + len, len >= 2 ? len - 2 : 0);
    std::fseek(f, 0L, SEEK_SET);
    std::memset(c, 0, sizeof c);
    if (!std::fgets(c, 300, f)) {
        std::fclose(f);
        return false;
    }
    out->seq.clear();
    char buf[1 << 16];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) {
        for (size_t i = 0; i < got; ++i) {
            const char b = buf[i];
            if (b == '\n' || b == '\r') continue;
            out->seq.push_back((unsigned char)b);
        }
    }
    std::fclose(f);
    return true;
}

}  // namespace swb
