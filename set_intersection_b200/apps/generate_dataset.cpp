// generate_dataset: the reference's dataset generator (src/generate_dataset.cpp)
// with the same flags, distributions and output files, made reproducible.
//
//   generate_dataset --universe U [--k 100] [--distribution uniform|normal|bernoulli|zipf]
//                    [--iterations 10000000] [--prob 0.5] [--stdev 2] [--skew 0.9]
//                    [--output out] [--seed 0] [--threads 0]
//
// Writes <output>_asc_<name> (sets by size, smallest first) and
// <output>_desc_<name> (largest first), where <name> is built as the reference
// builds it (src/generate_dataset.cpp:63-82): "<distribution>_<k>_<universe>"
// then "_<iterations>" (uniform), "_<iterations>_<stdev>" (normal), "_<prob>"
// (bernoulli) or "_<iterations>_<skew>" (zipf), then ".bin".
//
// Every set is a sorted set of distinct values of [1, universe]:
//  * uniform:   `iterations` uniform draws, repeats merged
//  * normal:    `iterations` draws of N(universe / 2, stdev), rounded to the
//               nearest integer; draws outside [1, universe] are dropped
//  * bernoulli: every value independently with probability prob (drawn as
//               geometric gaps between members)
//  * zipf:      `iterations` draws of Zipf(skew) over [1, universe]
//               (P(v) ~ v^-skew), repeats merged
//
// Differences from the reference, on purpose: set i draws from its own
// splitmix64 stream seeded by (--seed, i) instead of std::random_device, so a
// dataset can be regenerated, and the result does not depend on --threads;
// sets of equal size keep their index order in both files (a stable sort,
// where the reference's std::sort leaves ties unspecified); an unknown
// distribution is an error (the reference treats it as zipf); the uniform and
// zipf values are the drawn values (the reference shifts every drawn value up
// by one, src/generate_dataset.cpp:197-205, so its uniform sets can hold
// universe + 1, and its bitset has no bit for that value); normal draws outside
// the universe are dropped (the reference indexes its bitset with them).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <memory>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "si_random.hpp"

namespace {

struct Options {
    std::string output = "out", distribution = "uniform";
    uint64_t iterations = 10000000, seed = 0;
    double prob = 0.5, stdev = 2.0, skew = 0.9;
    uint64_t universe = 0;
    uint32_t k = 100;
    int threads = 0;
    bool help = false, has_universe = false;
};

bool parse_number(const std::string& s, double& v) {
    char* end = nullptr;
    v = std::strtod(s.c_str(), &end);
    return end && *end == '\0' && !s.empty();
}

bool parse_uint(const std::string& s, uint64_t& v) {
    if (s.empty() || s[0] == '-') return false;
    char* end = nullptr;
    v = std::strtoull(s.c_str(), &end, 10);
    return end && *end == '\0';
}

bool parse(int argc, char** argv, Options& o, std::string& why) {
    const std::map<std::string, int> flags = {{"distribution", 0}, {"output", 0}, {"prob", 1},     {"stdev", 1},
                                              {"skew", 1},         {"iterations", 2}, {"universe", 2}, {"k", 2},
                                              {"seed", 2},         {"threads", 2}};
    for (int i = 1; i < argc; ++i) {
        std::string s = argv[i];
        if (s == "--help") {
            o.help = true;
            continue;
        }
        if (s.rfind("--", 0) != 0) {
            why = "unexpected argument " + s;
            return false;
        }
        std::string key = s.substr(2), val;
        const size_t eq = key.find('=');
        if (eq != std::string::npos) {
            val = key.substr(eq + 1);
            key = key.substr(0, eq);
        } else if (i + 1 < argc) {
            val = argv[++i];
        } else {
            why = "Option '" + key + "' is missing an argument";
            return false;
        }
        auto it = flags.find(key);
        if (it == flags.end()) {
            why = "Option '" + key + "' does not exist";
            return false;
        }
        double d = 0;
        uint64_t u = 0;
        if (it->second == 1 && !parse_number(val, d)) {
            why = "Argument '" + val + "' failed to parse";
            return false;
        }
        if (it->second == 2 && !parse_uint(val, u)) {
            why = "Argument '" + val + "' failed to parse";
            return false;
        }
        if (key == "distribution") o.distribution = val;
        else if (key == "output") o.output = val;
        else if (key == "prob") o.prob = d;
        else if (key == "stdev") o.stdev = d;
        else if (key == "skew") o.skew = d;
        else if (key == "iterations") o.iterations = u;
        else if (key == "seed") o.seed = u;
        else if (key == "threads") o.threads = static_cast<int>(std::min<uint64_t>(u, 1024));
        else if (key == "k") {
            if (u > 0xffffffffull) {
                why = "k must fit 32 bits";
                return false;
            }
            o.k = static_cast<uint32_t>(u);
        } else if (key == "universe") {
            o.universe = u;
            o.has_universe = true;
        }
    }
    return true;
}

// Standard normal by the Box-Muller transform (one variate per pair of uniforms).
double normal01(si::Stream& rng) {
    double u1 = rng.uniform();
    while (u1 <= 0.0) u1 = rng.uniform();
    const double u2 = rng.uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

std::vector<uint32_t> make_set(const Options& o, uint32_t i, const si::Zipf* zipf) {
    si::Stream rng(si::mix64(o.seed * 0x9e3779b97f4a7c15ull + 0x2545f4914f6cdd1dull + i));
    const uint64_t U = o.universe;
    std::vector<uint32_t> s;
    if (o.distribution == "bernoulli") {
        if (o.prob <= 0.0 || U == 0) return s;
        if (o.prob >= 1.0) {
            s.resize(U);
            std::iota(s.begin(), s.end(), 1u);
            return s;
        }
        // gaps between members are geometric: P(gap = g) = (1 - p)^(g - 1) p
        const double lq = std::log1p(-o.prob);
        uint64_t v = 0;
        for (;;) {
            double u = rng.uniform();
            while (u <= 0.0) u = rng.uniform();
            const double g = std::floor(std::log(u) / lq) + 1.0;
            if (g > static_cast<double>(U - v)) break;
            v += static_cast<uint64_t>(g);
            s.push_back(static_cast<uint32_t>(v));
        }
        return s;
    }
    s.reserve(o.iterations);
    for (uint64_t it = 0; it < o.iterations; ++it) {
        if (o.distribution == "uniform") {
            s.push_back(static_cast<uint32_t>(1 + std::min<uint64_t>(U - 1, static_cast<uint64_t>(rng.uniform() * U))));
        } else if (o.distribution == "normal") {
            const double x = std::nearbyint(static_cast<double>(U / 2) + o.stdev * normal01(rng));
            if (x >= 1.0 && x <= static_cast<double>(U)) s.push_back(static_cast<uint32_t>(x));
        } else {
            s.push_back(static_cast<uint32_t>((*zipf)(rng)));
        }
    }
    std::sort(s.begin(), s.end());
    s.erase(std::unique(s.begin(), s.end()), s.end());
    return s;
}

bool write_dataset(const std::string& path, const std::vector<std::vector<uint32_t>>& sets,
                   const std::vector<uint32_t>& order, uint32_t universe, uint64_t total) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const uint32_t k = static_cast<uint32_t>(sets.size());
    bool ok = std::fwrite(&k, 4, 1, f) == 1 && std::fwrite(&universe, 4, 1, f) == 1 && std::fwrite(&total, 8, 1, f) == 1;
    for (uint32_t i : order) {
        const uint32_t n = static_cast<uint32_t>(sets[i].size());
        ok = ok && std::fwrite(&n, 4, 1, f) == 1;
    }
    for (uint32_t i : order) ok = ok && std::fwrite(sets[i].data(), 4, sets[i].size(), f) == sets[i].size();
    return std::fclose(f) == 0 && ok;
}

}  // namespace

int main(int argc, char** argv) {
    Options o;
    std::string why;
    if (!parse(argc, argv, o, why)) {
        std::printf("%s\n", why.c_str());
        return 1;
    }
    if (o.help) {
        std::printf(
            "Generate dataset\nUsage: %s --universe <U> [--k <sets>] [--distribution uniform|normal|bernoulli|zipf]\n"
            "  [--iterations <draws per set>] [--prob <p>] [--stdev <s>] [--skew <theta>] [--output <prefix>]\n"
            "  [--seed <n>] [--threads <n>]\n",
            argv[0]);
        return 0;
    }
    if (!o.has_universe) {
        std::printf("No universe given! Exiting...\n");
        return 1;
    }
    if (o.universe == 0 || o.universe > 0xffffffffull) {
        std::printf("universe must be in [1, 2^32 - 1]\n");
        return 1;
    }
    const std::string& dist = o.distribution;
    if (dist != "uniform" && dist != "normal" && dist != "bernoulli" && dist != "zipf") {
        std::printf("unknown distribution %s (uniform, normal, bernoulli or zipf)\n", dist.c_str());
        return 1;
    }
    if (dist == "bernoulli" && !(o.prob >= 0.0 && o.prob <= 1.0)) {
        std::printf("prob must be in [0, 1]\n");
        return 1;
    }
    if (dist == "zipf" && !(o.skew > 0.0)) {
        std::printf("skew must be positive\n");
        return 1;
    }

    std::string name = dist + "_" + std::to_string(o.k) + "_" + std::to_string(o.universe);
    if (dist == "uniform") name += "_" + std::to_string(o.iterations);
    else if (dist == "normal") name += "_" + std::to_string(o.iterations) + "_" + std::to_string(o.stdev);
    else if (dist == "bernoulli") name += "_" + std::to_string(o.prob);
    else name += "_" + std::to_string(o.iterations) + "_" + std::to_string(o.skew);
    name += ".bin";

    std::unique_ptr<si::Zipf> zipf;
    if (dist == "zipf") zipf.reset(new si::Zipf(o.universe, o.skew));
    std::vector<std::vector<uint32_t>> sets(o.k);
    unsigned T = o.threads > 0 ? static_cast<unsigned>(o.threads) : std::max(1u, std::thread::hardware_concurrency());
    T = std::max(1u, std::min<unsigned>(T, std::max<uint32_t>(o.k, 1u)));
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < T; ++t)
        pool.emplace_back([&, t] {
            for (uint32_t i = t; i < o.k; i += T) sets[i] = make_set(o, i, zipf.get());
        });
    for (auto& th : pool) th.join();
    uint64_t total = 0;
    for (auto& s : sets) total += s.size();

    std::vector<uint32_t> order(o.k);
    std::iota(order.begin(), order.end(), 0u);
    const uint32_t universe = static_cast<uint32_t>(o.universe);
    std::printf("Sorting sets in ascending order\n");
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return sets[a].size() < sets[b].size(); });
    std::string out = o.output + "_asc_" + name;
    std::printf("Writing dataset to %s\n", out.c_str());
    if (!write_dataset(out, sets, order, universe, total)) {
        std::printf("cannot write %s\n", out.c_str());
        return 1;
    }
    std::printf("Sorting sets in descending order\n");
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return sets[a].size() > sets[b].size(); });
    out = o.output + "_desc_" + name;
    std::printf("Writing dataset to %s\n", out.c_str());
    if (!write_dataset(out, sets, order, universe, total)) {
        std::printf("cannot write %s\n", out.c_str());
        return 1;
    }
    std::printf("Finished!\n");
    return 0;
}
