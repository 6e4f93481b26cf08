// app_common.hpp -- shared driver of the per-technique executables.
//
// Each executable of the reference (CMakeLists.txt:56-160: ip, obs, hi,
// bitmap_dynamic, bitmap_naive, matrix_multiplication) reads a binary dataset
// (include/io.hpp:25-54), counts the intersection of every pair of sets in
// runs of tile pairs (include/util.hpp:24-52, --partition), prints the dataset
// characteristics and its device timings, and with --output writes
// "(i,j): count" lines (include/io.hpp:91-136).  These executables take the
// same flags and write the same result file, calling libsi_b200.so for the
// counts.  Launch-geometry flags (--blocks, --threads, --warp, --path,
// --buckets, --bucket-size) are accepted and ignored: the engine sizes its own
// launches for the GPU it runs on.
//
// --output-binary <path> (an addition) also writes every count as binary:
// u32 k, u32 0, u64 C(k, 2), then the u32 counts of pairs (i, j), i < j, in
// row order (0,1), (0,2), ..., (0,k-1), (1,2), ... -- the triangular index of
// include/util.hpp:68-70 -- for loading into numpy or another tool without
// parsing text.
//
// Exit status: 0 on success, 1 on a flag or input error (as the reference),
// 2 on a device or library error (the reference exits with the CUDA error
// code, include/helpers.cuh:63-72).
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "si.h"

namespace si_app {

struct Dataset {
    uint32_t cardinality = 0, universe = 0;
    uint64_t total = 0;
    std::vector<uint32_t> sizes, elements;
    std::vector<uint64_t> offsets;  // k + 1
};

// Reads the reference's binary layout: u32 k, u32 universe, u64 total,
// u32 sizes[k], u32 elements[total]; checks it against the file size.
inline bool read_dataset(const std::string& path, Dataset& d, std::string& why) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
        why = "cannot open " + path;
        return false;
    }
    std::fseek(f, 0, SEEK_END);
    const long long fsize = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    bool ok = std::fread(&d.cardinality, 4, 1, f) == 1 && std::fread(&d.universe, 4, 1, f) == 1 &&
              std::fread(&d.total, 8, 1, f) == 1;
    const long long want = 16 + 4ll * d.cardinality + 4ll * static_cast<long long>(d.total);
    if (!ok || want != fsize) {
        std::fclose(f);
        why = "corrupt dataset header (sizes do not match the file)";
        return false;
    }
    d.sizes.resize(d.cardinality);
    d.elements.resize(d.total);
    ok = std::fread(d.sizes.data(), 4, d.cardinality, f) == d.cardinality &&
         std::fread(d.elements.data(), 4, d.total, f) == d.total;
    std::fclose(f);
    if (!ok) {
        why = "short read";
        return false;
    }
    d.offsets.assign(d.cardinality + 1, 0);
    for (uint32_t i = 0; i < d.cardinality; ++i) d.offsets[i + 1] = d.offsets[i] + d.sizes[i];
    if (d.offsets[d.cardinality] != d.total) {
        why = "set sizes do not add up to the element count";
        return false;
    }
    return true;
}

struct Tile {
    uint32_t id, start, end;
};

// include/util.hpp:24-52: tiles of `partition` sets, pairs (i, j >= i).
inline std::vector<std::pair<Tile, Tile>> tile_pairs(uint32_t k, uint32_t partition) {
    std::vector<Tile> tiles;
    const uint32_t n = (k + partition - 1) / partition;
    for (uint32_t i = 0; i < n; ++i) tiles.push_back({i, i * partition, std::min(k, (i + 1) * partition)});
    std::vector<std::pair<Tile, Tile>> runs;
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t j = i; j < n; ++j) runs.push_back({tiles[i], tiles[j]});
    return runs;
}

inline uint64_t tri(uint64_t n, uint64_t i, uint64_t j) { return n * (n - 1) / 2 - (n - i) * (n - i - 1) / 2 + j - i - 1; }

struct Args {
    std::string input, output, output_binary;
    uint32_t partition = 10000;
    bool help = false;
};

// --key value, --key=value, and bare boolean flags; unknown flags are errors.
inline bool parse_args(int argc, char** argv, const std::set<std::string>& value_flags,
                       const std::set<std::string>& bool_flags, Args& a, std::string& why) {
    for (int i = 1; i < argc; ++i) {
        std::string s = argv[i];
        if (s.rfind("--", 0) != 0) {
            why = "unexpected argument " + s;
            return false;
        }
        s = s.substr(2);
        std::string val;
        bool has_val = false;
        const size_t eq = s.find('=');
        if (eq != std::string::npos) {
            val = s.substr(eq + 1);
            s = s.substr(0, eq);
            has_val = true;
        }
        if (s == "help") {
            a.help = true;
            continue;
        }
        if (bool_flags.count(s)) continue;  // accepted, no effect (see header)
        if (!value_flags.count(s)) {
            why = "unknown option --" + s;
            return false;
        }
        if (!has_val) {
            if (i + 1 >= argc) {
                why = "option --" + s + " needs a value";
                return false;
            }
            val = argv[++i];
        }
        if (s == "input") {
            a.input = val;
        } else if (s == "output") {
            a.output = val;
        } else if (s == "output-binary") {
            a.output_binary = val;
        } else {
            char* end = nullptr;
            const unsigned long v = std::strtoul(val.c_str(), &end, 10);
            if (!end || *end || val.empty()) {
                why = "option --" + s + " needs a number";
                return false;
            }
            if (s == "partition") {
                if (v == 0) {
                    why = "--partition must be positive";
                    return false;
                }
                a.partition = static_cast<uint32_t>(v);
            }
        }
    }
    return true;
}

inline void box(const char* title, const std::vector<std::pair<std::string, std::string>>& rows) {
    std::printf("┌%s┐\n", title);
    for (auto& r : rows) std::printf("│%25s|%25s│\n", r.first.c_str(), r.second.c_str());
    std::printf("└───────────────────────────────────────────────────┘\n");
}

// Result text (include/io.hpp:91-136): "(i,j): count\n", 1-based, formatted by
// hand into a large buffer and written in big blocks.  Runs are formatted on
// a writer thread while the GPU computes the next run.
class ResultWriter {
  public:
    bool open(const std::string& path) {
        f_ = std::fopen(path.c_str(), "w");
        buf_.resize(kBuf);
        return f_ != nullptr;
    }
    ~ResultWriter() { close(); }
    void close() {
        join();
        if (f_) {
            flush();
            std::fclose(f_);
            f_ = nullptr;
        }
    }
    // all pairs of one run, in the reference's loop order; their counts are
    // rc[tri(k, i, j)] when k > 0 (the whole collection's triangle), else the
    // run's own layout (self: tri(stride, i - A, j - A), cross: (i - A) * stride + (j - B))
    void run_async(const Tile& A, const Tile& B, const uint32_t* rc, uint64_t stride, uint64_t k = 0) {
        join();
        worker_ = std::thread([this, A, B, rc, stride, k] {
            const bool self = A.id == B.id;
            for (uint32_t i = A.start; i < A.end; ++i)
                for (uint32_t j = self ? i + 1 : B.start; j < B.end; ++j)
                    line(i, j, rc[k ? tri(k, i, j)
                                    : self ? tri(stride, i - A.start, j - A.start)
                                           : uint64_t(i - A.start) * stride + (j - B.start)]);
        });
    }
    void join() {
        if (worker_.joinable()) worker_.join();
    }

  private:
    static constexpr size_t kBuf = 8u << 20;
    static char* put(char* p, uint32_t v) {
        char t[10];
        int n = 0;
        do {
            t[n++] = static_cast<char>('0' + v % 10);
            v /= 10;
        } while (v);
        while (n) *p++ = t[--n];
        return p;
    }
    void line(uint32_t i, uint32_t j, uint32_t c) {
        if (used_ + 48 > kBuf) flush();
        char* p = buf_.data() + used_;
        *p++ = '(';
        p = put(p, i + 1);
        *p++ = ',';
        p = put(p, j + 1);
        *p++ = ')';
        *p++ = ':';
        *p++ = ' ';
        p = put(p, c);
        *p++ = '\n';
        used_ = static_cast<size_t>(p - buf_.data());
    }
    void flush() {
        if (used_) std::fwrite(buf_.data(), 1, used_, f_);
        used_ = 0;
    }
    FILE* f_ = nullptr;
    std::vector<char> buf_;
    size_t used_ = 0;
    std::thread worker_;
};

enum class Kind { Sorted, Dense };

struct Spec {
    const char* name;         // executable name
    const char* banner;       // first line printed
    si_technique tech;        // engine technique
    Kind kind;
    std::set<std::string> value_flags, bool_flags;
};

#define SI_APP_TRY(expr)                                                                         \
    do {                                                                                         \
        const si_status st_ = (expr);                                                            \
        if (st_ != SI_OK) {                                                                      \
            std::fprintf(stderr, "%s: %s %s\n", #expr, si_status_string(st_), si_last_error_string()); \
            return 2;                                                                            \
        }                                                                                        \
    } while (0)

#define SI_APP_CUDA(expr)                                                                        \
    do {                                                                                         \
        const cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess) {                                                                 \
            std::fprintf(stderr, "%s: %s\n", #expr, cudaGetErrorString(e_));                     \
            return 2;                                                                            \
        }                                                                                        \
    } while (0)

inline int run(const Spec& spec, int argc, char** argv) {
    Args a;
    std::string why;
    std::set<std::string> vflags = spec.value_flags;
    vflags.insert("input");
    vflags.insert("output");
    vflags.insert("output-binary");
    if (!parse_args(argc, argv, vflags, spec.bool_flags, a, why)) {
        std::printf("%s\n", why.c_str());
        return 1;
    }
    if (a.help) {
        std::printf("%s\nUsage: %s --input <dataset> [--output <result>] [--output-binary <counts.bin>]", spec.banner,
                    spec.name);
        for (auto& f : spec.value_flags) std::printf(" [--%s <n>]", f.c_str());
        for (auto& f : spec.bool_flags) std::printf(" [--%s]", f.c_str());
        std::printf("\n");
        return 0;
    }
    if (a.input.empty()) {
        std::printf("No input dataset given! Exiting...\n");
        return 1;
    }
    std::printf("%s\n", spec.banner);
    Dataset d;
    if (!read_dataset(a.input, d, why)) {
        std::printf("%s: %s\n", a.input.c_str(), why.c_str());
        return 1;
    }
    box("──────────────Dataset characteristics──────────────",
        {{"Cardinality", std::to_string(d.cardinality)},
         {"Universe", std::to_string(d.universe)},
         {"Total elements", std::to_string(d.total)}});
    const uint32_t k = d.cardinality;
    const uint64_t pairs = uint64_t(k) * (k > 0 ? k - 1 : 0) / 2;
    std::vector<uint32_t> counts(pairs > 0 ? pairs : 1, 0);  // triangular order over the whole dataset
    std::vector<std::pair<std::string, double>> timings;
    auto t0 = std::chrono::steady_clock::now();
    auto lap = [&](const char* what) {
        auto t1 = std::chrono::steady_clock::now();
        timings.push_back({what, std::chrono::duration<double, std::milli>(t1 - t0).count()});
        t0 = t1;
    };

    uint32_t* d_el = nullptr;
    uint64_t* d_off = nullptr;
    SI_APP_CUDA(cudaMalloc(&d_el, std::max<uint64_t>(d.total, 1) * 4));
    SI_APP_CUDA(cudaMalloc(&d_off, (uint64_t(k) + 1) * 8));
    lap("Device memory allocation");
    SI_APP_CUDA(cudaMemcpy(d_el, d.elements.data(), d.total * 4, cudaMemcpyHostToDevice));
    SI_APP_CUDA(cudaMemcpy(d_off, d.offsets.data(), (uint64_t(k) + 1) * 8, cudaMemcpyHostToDevice));
    lap("Transfer to device");

    const auto runs = tile_pairs(k, a.partition);
    ResultWriter out;
    if (!a.output.empty()) {
        std::printf("Writing result to file %s\n", a.output.c_str());
        if (!out.open(a.output)) {
            std::printf("cannot write %s\n", a.output.c_str());
            return 1;
        }
    }
    bool streamed = false;  // the result lines were written run by run
    if (k == 2 && spec.kind == Kind::Sorted) {
        // one pair: the single-pair path
        const size_t ws_bytes = si_sisi_workspace_size(d.sizes[0], d.sizes[1], spec.tech);
        void* ws = nullptr;
        uint64_t* d_count = nullptr;
        SI_APP_CUDA(cudaMalloc(&ws, std::max<size_t>(ws_bytes, 256)));
        SI_APP_CUDA(cudaMalloc(&d_count, 8));
        SI_APP_TRY(si_sisi(d_el, d.sizes[0], d_el + d.offsets[1], d.sizes[1], spec.tech, d_count, nullptr, 0, ws,
                           ws_bytes, nullptr));
        SI_APP_TRY(si_workspace_check(ws, nullptr));
        uint64_t c = 0;
        SI_APP_CUDA(cudaMemcpy(&c, d_count, 8, cudaMemcpyDeviceToHost));
        counts[0] = static_cast<uint32_t>(c);
        lap("Intersection");
        cudaFree(ws);
        cudaFree(d_count);
    }
    bool dense_done = false;
    si_technique sorted_tech = spec.tech;
    if (k >= 2 && spec.kind == Kind::Dense) {
        // the whole triangle at once (the result lines follow the runs below)
        const size_t ws_bytes = si_misi_dense_workspace_size(k, d.universe, spec.tech);
        void* ws = nullptr;
        uint32_t* d_counts = nullptr;
        si_status st = SI_ERR_UNSUPPORTED;  // (workspace size 0: universe out of the dense range)
        if (ws_bytes) {
            SI_APP_CUDA(cudaMalloc(&ws, ws_bytes));
            SI_APP_CUDA(cudaMalloc(&d_counts, pairs * 4));
            st = si_misi_dense(d_el, d_off, k, d.universe, spec.tech, SI_DENSE_INT8, d_counts, ws, ws_bytes,
                               nullptr);
        }
        if (st == SI_ERR_UNSUPPORTED) {
            // a universe beyond the dense path's exact range: the same counts from the sorted sets
            std::printf("Universe %u is too large for the dense path; counting with bitmap_dynamic\n", d.universe);
            sorted_tech = SI_TECH_BITMAP;
        } else {
            SI_APP_TRY(st);
            SI_APP_TRY(si_workspace_check(ws, nullptr));
            lap("Intersection");
            SI_APP_CUDA(cudaMemcpy(counts.data(), d_counts, pairs * 4, cudaMemcpyDeviceToHost));
            lap("Transfer result");
            dense_done = true;
        }
        cudaFree(ws);
        cudaFree(d_counts);
    }
    if (k >= 2 && !dense_done && !(k == 2 && spec.kind == Kind::Sorted)) {
        // run by run, as the reference; each run's lines are formatted on the
        // writer thread while the next run computes (two host buffers)
        const uint32_t stride = runs.size() == 1 ? k : a.partition;
        const size_t ws_bytes = si_misi_workspace_size({0, std::min(k, a.partition)}, {0, std::min(k, a.partition)},
                                                       sorted_tech) +
                                si_misi_workspace_size({0, std::min(k, a.partition)},
                                                       {std::min(k, a.partition), std::min(k, 2 * a.partition)},
                                                       sorted_tech);
        const uint64_t run_counts = runs.size() == 1 ? pairs : uint64_t(stride) * stride;
        void* ws = nullptr;
        uint32_t* d_counts = nullptr;
        SI_APP_CUDA(cudaMalloc(&ws, ws_bytes));
        SI_APP_CUDA(cudaMalloc(&d_counts, run_counts * 4));
        std::vector<uint32_t> rc[2] = {std::vector<uint32_t>(run_counts), std::vector<uint32_t>(run_counts)};
        double t_int = 0, t_res = 0;
        int cur = 0;
        for (auto& run : runs) {
            const Tile& A = run.first;
            const Tile& B = run.second;
            auto r0 = std::chrono::steady_clock::now();
            SI_APP_TRY(si_misi(d_el, d_off, {A.start, A.end}, {B.start, B.end}, stride, sorted_tech, d_counts, ws,
                               ws_bytes, nullptr));
            SI_APP_TRY(si_workspace_check(ws, nullptr));
            auto r1 = std::chrono::steady_clock::now();
            SI_APP_CUDA(cudaMemcpy(rc[cur].data(), d_counts, run_counts * 4, cudaMemcpyDeviceToHost));
            auto r2 = std::chrono::steady_clock::now();
            if (!a.output_binary.empty()) {  // into the whole-collection triangle
                const bool self = A.id == B.id;
                for (uint32_t i = A.start; i < A.end; ++i)
                    for (uint32_t j = self ? i + 1 : B.start; j < B.end; ++j)
                        counts[tri(k, i, j)] = rc[cur][self ? tri(stride, i - A.start, j - A.start)
                                                            : uint64_t(i - A.start) * stride + (j - B.start)];
            }
            if (!a.output.empty()) {
                out.run_async(A, B, rc[cur].data(), stride);  // waits for the run before the previous one
                cur ^= 1;
            }
            t_int += std::chrono::duration<double, std::milli>(r1 - r0).count();
            t_res += std::chrono::duration<double, std::milli>(r2 - r1).count();
        }
        out.join();
        streamed = true;
        timings.push_back({"Intersection", t_int});
        timings.push_back({"Transfer result", t_res});
        t0 = std::chrono::steady_clock::now();
        cudaFree(ws);
        cudaFree(d_counts);
    }
    cudaFree(d_el);
    cudaFree(d_off);
    lap("Free device memory");

    std::vector<std::pair<std::string, std::string>> rows;
    double total = 0;
    char buf[64];
    for (auto& t : timings) {
        std::snprintf(buf, sizeof(buf), "%.3f", t.second);
        rows.push_back({t.first, buf});
        total += t.second;
    }
    std::snprintf(buf, sizeof(buf), "%.3f", total);
    rows.push_back({"Total", buf});
    box("────────────────Timings (in ms)────────────────────", rows);

    if (!a.output_binary.empty()) {
        FILE* f = std::fopen(a.output_binary.c_str(), "wb");
        const uint32_t zero = 0;
        bool ok = f && std::fwrite(&k, 4, 1, f) == 1 && std::fwrite(&zero, 4, 1, f) == 1 &&
                  std::fwrite(&pairs, 8, 1, f) == 1 && std::fwrite(counts.data(), 4, pairs, f) == pairs;
        if (f) ok = std::fclose(f) == 0 && ok;
        if (!ok) {
            std::printf("cannot write %s\n", a.output_binary.c_str());
            return 1;
        }
    }
    if (!a.output.empty()) {
        // the whole-collection counts (single pair, dense path) follow the
        // runs' order: a run is a self tile or a cross tile of the triangle
        if (!streamed && k >= 2) {
            for (auto& run : runs) {
                out.run_async(run.first, run.second, counts.data(), 0, k);
                out.join();
            }
        }
        out.close();
        std::printf("Finished\n");
    }
    return 0;
}

}  // namespace si_app
