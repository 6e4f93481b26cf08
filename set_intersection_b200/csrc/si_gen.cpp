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
#include <algorithm>
#include <cstdint>
#include <thread>
#include <unordered_set>
#include <vector>

#include "si.h"

namespace si {
namespace {

inline uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

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

}  // namespace
}  // namespace si

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
