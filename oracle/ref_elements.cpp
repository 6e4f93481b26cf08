// ref_elements -- materialised-intersection oracle built against the reference's
// own dataset reader.
//
// The reference's CPU executable src/std_set_intersection.cpp computes each
// pair's intersection with std::set_intersection into a vector v and keeps
// only v.size() (:68-73).  This driver reads a dataset with the reference's
// readDataset/datasetToCollection (include/io.hpp:25-68, compiled from where it
// lies) and writes, for the pair (set 0, set 1), the elements that same call
// produces, so element-level parity is pinned to the reference's data path.
//
// Output file (little-endian): u64 count, then count u32 elements.
// Usage: ref_elements <dataset.bin> <out.bin>
//
// Test infrastructure only (built into oracle/_ref/ by oracle/Makefile).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>
#include "io.hpp"

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <dataset.bin> <out.bin>\n", argv[0]);
        return 1;
    }
    std::string input = argv[1];
    Dataset* d = readDataset(input);
    if (d->cardinality < 2) {
        std::fprintf(stderr, "dataset needs at least 2 sets\n");
        return 1;
    }
    std::vector<std::vector<unsigned int>> sets = datasetToCollection(d);
    std::vector<unsigned int> v(std::min(sets[0].size(), sets[1].size()));
    auto it = std::set_intersection(sets[0].begin(), sets[0].end(), sets[1].begin(), sets[1].end(), v.begin());
    v.resize(it - v.begin());
    std::FILE* f = std::fopen(argv[2], "wb");
    if (!f) return 1;
    std::uint64_t n = v.size();
    std::fwrite(&n, sizeof(n), 1, f);
    if (n) std::fwrite(v.data(), sizeof(unsigned int), n, f);
    std::fclose(f);
    return 0;
}
