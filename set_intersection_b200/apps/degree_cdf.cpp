// degree_cdf: the reference's dataset statistics tool (src/degree_cdf.cpp):
//
//   degree_cdf <dataset.bin> <prefix> [--device]
//
// writes four text files of "first second" lines:
//   <prefix>_degree_set.txt      (set size, 1-based set id), by set size
//   <prefix>_degree_element.txt  (inverted-list length, value), by length, for
//                                every value 0 .. universe - 1
//   <prefix>_set_cdf.txt         (set size, running sum over the sets taken in
//                                size order of the summed inverted-list lengths
//                                of each set's values), by set size
//   <prefix>_element_cdf.txt     (inverted-list length L, running sum of L^2),
//                                by length
// Orders among equal keys follow std::sort with the reference's comparators on
// the same input sequences, so the first three files are byte-identical to
// the reference's.  Differences, on purpose: _element_cdf.txt holds the element
// CDF (the reference computes it but writes the set CDF into that file,
// src/degree_cdf.cpp:85-86); and when the dataset holds the value `universe`
// itself, the inverted index gets a slot for it (the reference sizes the index
// `universe` and then writes past its end, src/degree_cdf.cpp:22), so
// degree_element has a line for that value too.  Counts are 64-bit (the
// reference's per-set sum is 32-bit).  With --device the inverted-list
// lengths and the per-set sums come from si_degree_stats on the GPU; the
// sorts and running sums are the same host code either way.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <string>
#include <utility>
#include <vector>

#include "app_common.hpp"

namespace {

template <class T>
bool write_pairs(const std::vector<T>& pairs, const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    for (auto& p : pairs)
        std::fprintf(f, "%llu %llu\n", static_cast<unsigned long long>(p.first),
                     static_cast<unsigned long long>(p.second));
    return std::fclose(f) == 0;
}

}  // namespace

// inv[v] and the per-set sums through the library, on the GPU.
int device_stats(const si_app::Dataset& d, uint64_t slots, std::vector<uint64_t>& inv, std::vector<uint64_t>& sums) {
    const uint32_t k = d.cardinality;
    uint32_t *d_el = nullptr, *d_inv = nullptr;
    uint64_t *d_off = nullptr, *d_sum = nullptr;
    void* ws = nullptr;
    const size_t ws_bytes = si_degree_stats_workspace_size();
    SI_APP_CUDA(cudaMalloc(&d_el, std::max<uint64_t>(d.total, 1) * 4));
    SI_APP_CUDA(cudaMalloc(&d_off, (uint64_t(k) + 1) * 8));
    SI_APP_CUDA(cudaMalloc(&d_inv, std::max<uint64_t>(slots, 1) * 4));
    SI_APP_CUDA(cudaMalloc(&d_sum, std::max<uint64_t>(k, 1) * 8));
    SI_APP_CUDA(cudaMalloc(&ws, ws_bytes));
    SI_APP_CUDA(cudaMemcpy(d_el, d.elements.data(), d.total * 4, cudaMemcpyHostToDevice));
    SI_APP_CUDA(cudaMemcpy(d_off, d.offsets.data(), (uint64_t(k) + 1) * 8, cudaMemcpyHostToDevice));
    SI_APP_TRY(si_degree_stats(d_el, d_off, k, d.total, slots, d_inv, d_sum, ws, ws_bytes, nullptr));
    SI_APP_TRY(si_workspace_check(ws, nullptr));
    std::vector<uint32_t> inv32(slots);
    sums.assign(k, 0);
    SI_APP_CUDA(cudaMemcpy(inv32.data(), d_inv, slots * 4, cudaMemcpyDeviceToHost));
    SI_APP_CUDA(cudaMemcpy(sums.data(), d_sum, uint64_t(k) * 8, cudaMemcpyDeviceToHost));
    inv.assign(inv32.begin(), inv32.end());
    cudaFree(d_el);
    cudaFree(d_off);
    cudaFree(d_inv);
    cudaFree(d_sum);
    cudaFree(ws);
    return 0;
}

int main(int argc, char** argv) {
    const bool on_device = argc == 4 && std::string(argv[3]) == "--device";
    if (argc != 3 && !on_device) {
        std::printf("Usage: %s <dataset.bin> <output prefix> [--device]\n", argv[0]);
        return 1;
    }
    si_app::Dataset d;
    std::string why;
    if (!si_app::read_dataset(argv[1], d, why)) {
        std::printf("%s: %s\n", argv[1], why.c_str());
        return 1;
    }
    uint32_t vmax = 0;
    for (uint64_t e = 0; e < d.total; ++e) vmax = std::max(vmax, d.elements[e]);
    if (d.total && vmax > d.universe) {
        std::printf("%s: value %u above the universe %u\n", argv[1], vmax, d.universe);
        return 1;
    }
    // one slot per value 0 .. universe - 1, and one for `universe` when it occurs
    const uint64_t slots = uint64_t(d.universe) + (d.total && vmax == d.universe ? 1 : 0);
    // inverted-list lengths (how many sets hold each value) and, per set,
    // the sum of its values' lengths
    std::vector<uint64_t> inv, sums;
    if (on_device) {
        if (const int rc = device_stats(d, slots, inv, sums)) return rc;
    } else {
        inv.assign(slots, 0);
        for (uint64_t e = 0; e < d.total; ++e) ++inv[d.elements[e]];
        sums.assign(d.cardinality, 0);
        for (uint32_t s = 0; s < d.cardinality; ++s)
            for (uint64_t e = d.offsets[s]; e < d.offsets[s + 1]; ++e) sums[s] += inv[d.elements[e]];
    }
    using P32 = std::pair<unsigned int, unsigned int>;
    using P64 = std::pair<unsigned long long, unsigned long long>;
    std::vector<P32> degree_set;
    std::vector<P64> set_cdf;
    for (uint32_t s = 0; s < d.cardinality; ++s) {
        degree_set.emplace_back(d.sizes[s], s + 1);
        set_cdf.emplace_back(d.sizes[s], sums[s]);
    }
    std::vector<P32> degree_element;
    std::vector<P64> element_cdf;
    for (uint64_t v = 0; v < slots; ++v) {
        element_cdf.emplace_back(inv[v], inv[v]);
        degree_element.emplace_back(static_cast<unsigned int>(inv[v]), static_cast<unsigned int>(v));
    }
    std::sort(degree_set.begin(), degree_set.end(), [](const P32& a, const P32& b) { return a.first < b.first; });
    std::sort(degree_element.begin(), degree_element.end(),
              [](const P32& a, const P32& b) { return a.first < b.first; });
    std::sort(set_cdf.begin(), set_cdf.end(), [](const P64& a, const P64& b) { return a.first < b.first; });
    std::sort(element_cdf.begin(), element_cdf.end(), [](const P64& a, const P64& b) { return a.first < b.first; });
    for (size_t i = 0; i < element_cdf.size(); ++i)
        element_cdf[i].second = (i ? element_cdf[i - 1].second : 0) + element_cdf[i].second * element_cdf[i].second;
    for (size_t i = 1; i < set_cdf.size(); ++i) set_cdf[i].second += set_cdf[i - 1].second;

    const std::string prefix = argv[2];
    const bool ok = write_pairs(degree_set, prefix + "_degree_set.txt") &&
                    write_pairs(degree_element, prefix + "_degree_element.txt") &&
                    write_pairs(set_cdf, prefix + "_set_cdf.txt") &&
                    write_pairs(element_cdf, prefix + "_element_cdf.txt");
    if (!ok) {
        std::printf("cannot write %s_*.txt\n", prefix.c_str());
        return 1;
    }
    std::printf("Finished\n");
    return 0;
}
