// txt2bin: drop-in for the reference's txt2bin (src/txt2bin.cpp:12-39):
//   txt2bin <sets.txt> <prefix>  ->  <prefix>_asc.bin (sets in file order) and
//                                    <prefix>_desc.bin (sets by size, largest first)
// One set per line, elements separated by spaces; the universe is the largest
// element.  Unlike the reference (which trusts its input), every set is checked
// to be strictly increasing and every token to be a 32-bit unsigned number;
// a bad line is reported and the exit status is 1.  Sets of equal size keep
// their file order in the _desc file (a stable sort).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

static bool write_bin(const std::string& path, const std::vector<std::vector<uint32_t>>& sets,
                      const std::vector<size_t>& order, uint32_t universe, uint64_t total) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const uint32_t k = static_cast<uint32_t>(sets.size());
    std::fwrite(&k, 4, 1, f);
    std::fwrite(&universe, 4, 1, f);
    std::fwrite(&total, 8, 1, f);
    for (size_t i : order) {
        const uint32_t n = static_cast<uint32_t>(sets[i].size());
        std::fwrite(&n, 4, 1, f);
    }
    for (size_t i : order) std::fwrite(sets[i].data(), 4, sets[i].size(), f);
    return std::fclose(f) == 0;
}

int main(int argc, char** argv) {
    if (argc != 3) {
        std::printf("Usage: %s <sets.txt> <output prefix>\n", argv[0]);
        return 1;
    }
    std::ifstream in(argv[1]);
    if (!in) {
        std::printf("cannot open %s\n", argv[1]);
        return 1;
    }
    std::vector<std::vector<uint32_t>> sets;
    uint32_t universe = 0;
    uint64_t total = 0, lineno = 0;
    std::string line, tok;
    while (std::getline(in, line)) {
        ++lineno;
        std::istringstream ss(line);
        std::vector<uint32_t> s;
        while (ss >> tok) {
            char* end = nullptr;
            const unsigned long long v = std::strtoull(tok.c_str(), &end, 10);
            if (!end || *end || v > 0xffffffffull || tok[0] == '-') {
                std::printf("%s:%llu: not a 32-bit unsigned number: %s\n", argv[1], (unsigned long long)lineno,
                            tok.c_str());
                return 1;
            }
            if (!s.empty() && v <= s.back()) {
                std::printf("%s:%llu: set is not strictly increasing at %s\n", argv[1], (unsigned long long)lineno,
                            tok.c_str());
                return 1;
            }
            s.push_back(static_cast<uint32_t>(v));
        }
        if (s.empty()) continue;  // blank lines are skipped, as in the reference
        universe = std::max(universe, s.back());
        total += s.size();
        sets.push_back(std::move(s));
    }
    std::vector<size_t> order(sets.size());
    std::iota(order.begin(), order.end(), 0);
    const std::string asc = std::string(argv[2]) + "_asc.bin", desc = std::string(argv[2]) + "_desc.bin";
    std::printf("Writing dataset to %s\n", asc.c_str());
    if (!write_bin(asc, sets, order, universe, total)) return 1;
    std::printf("Sorting sets in descending order\n");
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return sets[a].size() > sets[b].size(); });
    std::printf("Writing dataset to %s\n", desc.c_str());
    if (!write_bin(desc, sets, order, universe, total)) return 1;
    return 0;
}
