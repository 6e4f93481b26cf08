// bin2txt: drop-in for the reference's bin2txt (src/bin2txt.cpp:10-37):
//   bin2txt <dataset.bin> <prefix>  ->  <prefix>.txt, one set per line, each
//   element followed by a space.  The binary file is checked against its
//   header (exit status 1 on a truncated or inconsistent file).
#include <cstdio>
#include <string>

#include "app_common.hpp"

int main(int argc, char** argv) {
    if (argc != 3) {
        std::printf("Usage: %s <dataset.bin> <output prefix>\n", argv[0]);
        return 1;
    }
    si_app::Dataset d;
    std::string why;
    if (!si_app::read_dataset(argv[1], d, why)) {
        std::printf("%s: %s\n", argv[1], why.c_str());
        return 1;
    }
    const std::string out = std::string(argv[2]) + ".txt";
    std::printf("Writing dataset to %s\n", out.c_str());
    FILE* f = std::fopen(out.c_str(), "w");
    if (!f) return 1;
    std::vector<char> buf;
    buf.reserve(1u << 20);
    for (uint32_t i = 0; i < d.cardinality; ++i) {
        buf.clear();
        char tmp[12];
        for (uint64_t x = d.offsets[i]; x < d.offsets[i + 1]; ++x) {
            const int n = std::snprintf(tmp, sizeof(tmp), "%u ", d.elements[x]);
            buf.insert(buf.end(), tmp, tmp + n);
        }
        buf.push_back('\n');
        std::fwrite(buf.data(), 1, buf.size(), f);
    }
    return std::fclose(f) == 0 ? 0 : 1;
}
