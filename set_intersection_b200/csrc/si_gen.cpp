// si_gen.cpp -- seeded, deterministic host generators of sorted unique uint32
// sets (the engine's stand-in for src/generate_dataset.cpp, which seeds from
// std::random_device and so cannot reproduce a dataset).
//
// Uniform without replacement, exactly n values from [lo, hi):
//  * dense case (n > U/64): every candidate v gets the key
//    (hash32(seed, v) << 32 | (v - lo)); the n smallest keys are selected by a
//    two-level radix select on the hash, then emitted in increasing v, so the
//    result is a uniformly random n-subset, already sorted.  The result does
//    not depend on the thread count.
//  * sparse case: sequential draws from a splitmix64 stream, rejecting
//    repeats until n distinct values are held, then sorted (the classic
//    draw-until-distinct construction of a uniform n-subset).
//
// Bernoulli membership (a dense collection): value v is in set a iff
// hash32(seed, a * 2^32 + v) < p * 2^32, independently for every (a, v).
//
// Log-uniform pool: sizes log-uniform on [n_min, n_max]; each set n distinct
// uniform values of [0, universe).
//
// Power-law collection: set sizes from the continuous power law
// P(n) ~ n^-size_exp on [n_min, n_max + 1), floored (inverse-CDF sampling);
// each set then holds that many DISTINCT values of [1, universe] drawn with
// Zipf popularity P(v) ~ v^-value_exp by rejection-inversion sampling
// (Hormann and Derflinger, "Rejection-inversion to generate variates from
// monotone discrete distributions", 1996), repeats rejected.  Every set has
// its own random stream (splitmix64 of seed and set index), so the result
// does not depend on the thread count.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <unordered_set>
#include <vector>

#include "si.h"
#include "si_random.hpp"

namespace si {
namespace {

inline uint32_t hash32(uint64_t seed, uint64_t v) {
    return static_cast<uint32_t>(mix64(v + seed * 0x9e3779b97f4a7c15ull + 0x632be59bd9b4e019ull) >> 32);
}

int resolve_threads(int threads) {
    if (threads > 0) return threads;
    unsigned hc = std::thread::hardware_concurrency();
    return hc ? static_cast<int>(std::min(hc, 256u)) : 1;
}

template <class F>
void parallel_chunks(uint64_t n, int T, F&& f) {  // f(thread, begin, end)
    std::vector<std::thread> pool;
    for (int t = 0; t < T; ++t) {
        uint64_t b = n * t / T, e = n * (t + 1) / T;
        pool.emplace_back([&f, t, b, e] { f(t, b, e); });
    }
    for (auto& th : pool) th.join();
}

void uniform_dense(uint64_t seed, uint64_t n, uint64_t lo, uint64_t U, uint32_t* out, int T) {
    // Pass 1: histogram of the hash's top 16 bits.
    std::vector<std::vector<uint64_t>> h(T, std::vector<uint64_t>(65536, 0));
    parallel_chunks(U, T, [&](int t, uint64_t b, uint64_t e) {
        auto& H = h[t];
        for (uint64_t v = b; v < e; ++v) ++H[hash32(seed, lo + v) >> 16];
    });
    uint64_t need = n, bin1 = 0;
    for (; bin1 < 65536; ++bin1) {
        uint64_t c = 0;
        for (int t = 0; t < T; ++t) c += h[t][bin1];
        if (c >= need) break;
        need -= c;
    }
    // Pass 2: histogram of the low 16 bits inside that bin.
    for (auto& H : h) std::fill(H.begin(), H.end(), 0);
    parallel_chunks(U, T, [&](int t, uint64_t b, uint64_t e) {
        auto& H = h[t];
        for (uint64_t v = b; v < e; ++v) {
            uint32_t x = hash32(seed, lo + v);
            if ((x >> 16) == bin1) ++H[x & 0xffff];
        }
    });
    uint64_t bin2 = 0;
    for (; bin2 < 65536; ++bin2) {
        uint64_t c = 0;
        for (int t = 0; t < T; ++t) c += h[t][bin2];
        if (c >= need) break;
        need -= c;
    }
    const uint32_t thr = static_cast<uint32_t>((bin1 << 16) | bin2);
    // `need` values with hash == thr are taken, the smallest v first.
    // Pass 3: per-chunk counts of (hash < thr) and (hash == thr).
    std::vector<uint64_t> below(T, 0), equal(T, 0);
    parallel_chunks(U, T, [&](int t, uint64_t b, uint64_t e) {
        uint64_t c0 = 0, c1 = 0;
        for (uint64_t v = b; v < e; ++v) {
            uint32_t x = hash32(seed, lo + v);
            c0 += x < thr;
            c1 += x == thr;
        }
        below[t] = c0;
        equal[t] = c1;
    });
    std::vector<uint64_t> pos(T, 0), eq_before(T, 0);
    uint64_t acc = 0, eacc = 0;
    for (int t = 0; t < T; ++t) {
        pos[t] = acc;
        eq_before[t] = eacc;
        uint64_t take_eq = eacc >= need ? 0 : std::min(equal[t], need - eacc);
        acc += below[t] + take_eq;
        eacc += equal[t];
    }
    // Pass 4: emit in increasing v.
    parallel_chunks(U, T, [&](int t, uint64_t b, uint64_t e) {
        uint64_t p = pos[t], eseen = eq_before[t];
        for (uint64_t v = b; v < e; ++v) {
            uint32_t x = hash32(seed, lo + v);
            if (x < thr) {
                out[p++] = static_cast<uint32_t>(lo + v);
            } else if (x == thr) {
                if (eseen < need) out[p++] = static_cast<uint32_t>(lo + v);
                ++eseen;
            }
        }
    });
}

void uniform_sparse(uint64_t seed, uint64_t n, uint64_t lo, uint64_t U, uint32_t* out) {
    std::unordered_set<uint32_t> seen;
    seen.reserve(n * 2);
    uint64_t state = seed * 0x9e3779b97f4a7c15ull + 0x2545f4914f6cdd1dull;
    uint64_t k = 0;
    while (k < n) {
        state += 0x9e3779b97f4a7c15ull;
        const uint64_t r = mix64(state);
        const uint32_t v = static_cast<uint32_t>(lo + static_cast<uint64_t>((static_cast<unsigned __int128>(r) * U) >> 64));
        if (seen.insert(v).second) out[k++] = v;
    }
    std::sort(out, out + n);
}

uint64_t powerlaw_size(uint64_t seed, uint64_t a, uint32_t n_min, uint32_t n_max, double e) {
    Stream rng(mix64(seed * 0x2545f4914f6cdd1dull + a));
    const double u = rng.uniform();
    const double lo = n_min, hi = static_cast<double>(n_max) + 1.0;
    double x;
    if (std::fabs(e - 1.0) < 1e-12) {
        x = lo * std::exp(u * std::log(hi / lo));
    } else {
        const double q = 1.0 - e;
        x = std::pow(std::pow(lo, q) + u * (std::pow(hi, q) - std::pow(lo, q)), 1.0 / q);
    }
    const uint64_t n = static_cast<uint64_t>(std::floor(x));
    return std::min<uint64_t>(std::max<uint64_t>(n, n_min), n_max);
}

}  // namespace
}  // namespace si

extern "C" si_status si_gen_loguniform(uint64_t seed, uint32_t k, uint32_t n_min, uint32_t n_max, uint32_t universe,
                                       uint64_t* offsets, uint32_t* elements, int threads) {
    if (!offsets || n_min == 0 || n_min > n_max || static_cast<uint64_t>(n_max) * 2 > universe)
        return SI_ERR_INVALID_ARGUMENT;
    const int T = si::resolve_threads(threads);
    if (!elements) {
        offsets[0] = 0;
        const double l0 = std::log(static_cast<double>(n_min)), l1 = std::log(static_cast<double>(n_max) + 1.0);
        si::parallel_chunks(k, T, [&](int, uint64_t b, uint64_t e) {
            for (uint64_t a = b; a < e; ++a) {
                si::Stream rng(si::mix64(seed * 0x2545f4914f6cdd1dull + 0x3c6ef372fe94f82bull + a));
                const uint64_t n = static_cast<uint64_t>(std::floor(std::exp(l0 + rng.uniform() * (l1 - l0))));
                offsets[a + 1] = std::min<uint64_t>(std::max<uint64_t>(n, n_min), n_max);
            }
        });
        for (uint32_t a = 0; a < k; ++a) offsets[a + 1] += offsets[a];
        return SI_OK;
    }
    // n distinct values of [0, universe): n draws, sort, unique, and more draws
    // for the few repeats until n are held
    si::parallel_chunks(k, T, [&](int, uint64_t b, uint64_t e) {
        std::vector<uint32_t> v;
        for (uint64_t a = b; a < e; ++a) {
            const uint64_t n = offsets[a + 1] - offsets[a];
            si::Stream rng(si::mix64(seed * 0x9e3779b97f4a7c15ull + 0x7f4a7c159e3779b9ull + a));
            v.clear();
            while (v.size() < n) {
                const size_t need = n - v.size();
                for (size_t i = 0; i < need; ++i)
                    v.push_back(static_cast<uint32_t>((static_cast<unsigned __int128>(rng.next()) * universe) >> 64));
                std::sort(v.begin(), v.end());
                v.erase(std::unique(v.begin(), v.end()), v.end());
            }
            std::copy(v.begin(), v.end(), elements + offsets[a]);
        }
    });
    return SI_OK;
}

extern "C" si_status si_gen_powerlaw(uint64_t seed, uint32_t k, uint32_t n_min, uint32_t n_max, double size_exp,
                                     uint32_t universe, double value_exp, uint64_t* offsets, uint32_t* elements,
                                     int threads) {
    if (!offsets || n_min == 0 || n_min > n_max || n_max > universe || !(size_exp > 0.0) || !(value_exp >= 0.0))
        return SI_ERR_INVALID_ARGUMENT;
    const int T = si::resolve_threads(threads);
    if (!elements) {
        offsets[0] = 0;
        si::parallel_chunks(k, T, [&](int, uint64_t b, uint64_t e) {
            for (uint64_t a = b; a < e; ++a) offsets[a + 1] = si::powerlaw_size(seed, a, n_min, n_max, size_exp);
        });
        for (uint32_t a = 0; a < k; ++a) offsets[a + 1] += offsets[a];
        return SI_OK;
    }
    const si::Zipf zipf(universe, value_exp);
    si::parallel_chunks(k, T, [&](int, uint64_t b, uint64_t e) {
        std::vector<uint64_t> seen((static_cast<uint64_t>(universe) >> 6) + 1);
        for (uint64_t a = b; a < e; ++a) {
            const uint64_t n = offsets[a + 1] - offsets[a];
            si::Stream rng(si::mix64(seed * 0x9e3779b97f4a7c15ull + 0x51ed270b2da3ab9bull + a));
            std::vector<uint32_t> vals;
            vals.reserve(n);
            while (vals.size() < n) {
                const uint64_t v = zipf(rng);
                uint64_t& w = seen[v >> 6];
                if (w & (1ull << (v & 63))) continue;
                w |= 1ull << (v & 63);
                vals.push_back(static_cast<uint32_t>(v));
            }
            for (uint32_t v : vals) seen[v >> 6] &= ~(1ull << (v & 63));
            std::sort(vals.begin(), vals.end());
            std::copy(vals.begin(), vals.end(), elements + offsets[a]);
        }
    });
    return SI_OK;
}

extern "C" si_status si_gen_bernoulli(uint64_t seed, uint32_t k, uint32_t n_values, double p, uint64_t* offsets,
                                      uint32_t* elements, int threads) {
    if (!offsets || !(p >= 0.0 && p <= 1.0)) return SI_ERR_INVALID_ARGUMENT;
    const uint64_t thr = static_cast<uint64_t>(p * 4294967296.0);  // member iff hash < thr
    const int T = si::resolve_threads(threads);
    auto member = [&](uint64_t a, uint64_t v) { return si::hash32(seed, (a << 32) | v) < thr; };
    if (!elements) {
        offsets[0] = 0;
        si::parallel_chunks(k, T, [&](int, uint64_t b, uint64_t e) {
            for (uint64_t a = b; a < e; ++a) {
                uint64_t c = 0;
                for (uint64_t v = 0; v < n_values; ++v) c += member(a, v);
                offsets[a + 1] = c;
            }
        });
        for (uint32_t a = 0; a < k; ++a) offsets[a + 1] += offsets[a];
        return SI_OK;
    }
    si::parallel_chunks(k, T, [&](int, uint64_t b, uint64_t e) {
        for (uint64_t a = b; a < e; ++a) {
            uint64_t x = offsets[a];
            for (uint64_t v = 0; v < n_values; ++v)
                if (member(a, v)) elements[x++] = static_cast<uint32_t>(v);
        }
    });
    return SI_OK;
}

extern "C" si_status si_gen_uniform(uint64_t seed, uint64_t n, uint64_t lo, uint64_t hi, uint32_t* out, int threads) {
    if (hi < lo || hi - lo > (1ull << 32) || hi > (1ull << 32) || n > hi - lo || (n && !out))
        return SI_ERR_INVALID_ARGUMENT;
    if (n == 0) return SI_OK;
    const uint64_t U = hi - lo;
    if (n > U / 64) si::uniform_dense(seed, n, lo, U, out, si::resolve_threads(threads));
    else si::uniform_sparse(seed, n, lo, U, out);
    return SI_OK;
}
