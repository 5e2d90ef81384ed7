// fasta.h -- the reference's single-record FASTA reader (src/FASTA.cpp:39-86).
#pragma once

#include <string>
#include <vector>

namespace swb {

struct FastaRecord {
    std::string name;           // header without '>' and its last character
    std::vector<unsigned char> seq;
};

// Same acceptance rules as FASTAsequence::load: the file must open and its first
// character must be '>'; the first line (up to 299 bytes) is the header, every
// other byte except '\n' and '\r' is sequence, kept as it is (no case folding,
// no alphabet).  Returns false when the reference would fail the load.
bool fasta_load(const char *path, FastaRecord *out);

}  // namespace swb
