/*
 * si_oracle.c -- CPU restatement of chribell/set_intersection's CPU techniques.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: it is loaded by tests/,
 * by __graft_entry__.smoke() and by bench.py's cpu_baseline / reference legs.
 * The product library (set_intersection_b200) never links, loads or calls it.
 *
 * Parity pin: tests/test_oracle.py checks every function here against golden
 * result files written by the reference's own CPU executables
 * (stdintersection, serial_intersect, boost_bitset built from the reference
 * sources by oracle/Makefile into oracle/_ref/), see tests/golden/make_golden.py.
 *
 * Functions follow (paths relative to the reference repository):
 *   si_oracle_set_intersection  <- src/std_set_intersection.cpp:68-73 (std::set_intersection,
 *                                  elements materialised into v, count = v.size())
 *   si_oracle_serial_intersect  <- src/serial_intersect.cpp:93-113 (two-pointer count)
 *   si_oracle_all_pairs         <- the OpenMP pair loops of src/std_set_intersection.cpp:58-76,
 *                                  src/serial_intersect.cpp:61-76, src/boost_bitset.cpp:60-84
 *   si_oracle_triangular_index  <- include/util.hpp:68-70
 *   si_oracle_gen_uniform       <- no reference counterpart: the engine's seeded input
 *                                  generator restated, so that the reference's executables
 *                                  read the very sets the engine is timed on
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

uint64_t si_oracle_triangular_index(uint64_t n, uint64_t i, uint64_t j)
{
    /* include/util.hpp:68-70: offset of pair (i<j) in the row-major upper triangle. */
    return (n * (n - 1) / 2) - (n - i) * ((n - i) - 1) / 2 + j - i - 1;
}

uint64_t si_oracle_combination2(uint64_t n)
{
    return n < 2 ? 0 : n * (n - 1) / 2;
}

/* std::set_intersection on two ascending ranges: advance the smaller head,
 * emit on equality and advance both.  out may be NULL (count only). */
uint64_t si_oracle_set_intersection(const uint32_t* a, uint64_t na,
                                    const uint32_t* b, uint64_t nb, uint32_t* out)
{
    uint64_t i = 0, j = 0, c = 0;
    while (i < na && j < nb) {
        if (a[i] < b[j]) {
            ++i;
        } else if (b[j] < a[i]) {
            ++j;
        } else {
            if (out) out[c] = a[i];
            ++c; ++i; ++j;
        }
    }
    return c;
}

/* serialIntersect of src/serial_intersect.cpp:93-113: equality first, then the
 * smaller side advances. */
uint64_t si_oracle_serial_intersect(const uint32_t* a, uint64_t na,
                                    const uint32_t* b, uint64_t nb)
{
    uint64_t i = 0, j = 0, c = 0;
    while (i < na && j < nb) {
        if (a[i] == b[j]) { ++i; ++j; ++c; }
        else if (a[i] < b[j]) { ++i; }
        else { ++j; }
    }
    return c;
}

enum { SI_ORACLE_STD = 0, SI_ORACLE_SERIAL = 1, SI_ORACLE_BITSET = 2 };

/* Bitset probe of src/boost_bitset.cpp:69-83: a bitset of universe+1 bits holds
 * set a (the reference does universe++ at :49 before sizing), every later set b
 * is probed element by element. */
static void bitset_row(const uint32_t* elements, const uint64_t* offsets, uint32_t k,
                       uint32_t a, uint64_t* bits, uint64_t nwords, uint32_t* counts)
{
    memset(bits, 0, nwords * sizeof(uint64_t));
    for (uint64_t x = offsets[a]; x < offsets[a + 1]; ++x) {
        uint32_t e = elements[x];
        bits[e >> 6] |= 1ull << (e & 63);
    }
    for (uint32_t b = a + 1; b < k; ++b) {
        uint32_t c = 0;
        for (uint64_t x = offsets[b]; x < offsets[b + 1]; ++x) {
            uint32_t e = elements[x];
            c += (uint32_t)((bits[e >> 6] >> (e & 63)) & 1ull);
        }
        counts[si_oracle_triangular_index(k, a, b)] = c;
    }
}

/* All pairs a<b of a CSR collection (offsets has k+1 entries), counts in the
 * triangular layout.  threads <= 0 means "all available".  The work split is
 * the reference's: thread t takes a in [k*t/T, k*(t+1)/T)
 * (src/std_set_intersection.cpp:62-64).  Returns 0, or -1 on a bad argument. */
int si_oracle_all_pairs(const uint32_t* elements, const uint64_t* offsets, uint32_t k,
                        uint32_t universe, int technique, int threads, uint32_t* counts)
{
    if (technique < 0 || technique > 2) return -1;
    if (k < 2) return 0;
#ifdef _OPENMP
    int T = threads > 0 ? threads : omp_get_max_threads();
#else
    int T = 1;
    (void)threads;
#endif
    uint64_t nwords = ((uint64_t)universe + 1 + 63) / 64;
    int bad = 0;
#ifdef _OPENMP
#pragma omp parallel num_threads(T) reduction(|:bad)
#endif
    {
#ifdef _OPENMP
        int t = omp_get_thread_num();
#else
        int t = 0;
#endif
        uint32_t lower = (uint32_t)((uint64_t)k * t / T);
        uint32_t upper = (uint32_t)((uint64_t)k * (t + 1) / T);
        uint64_t* bits = NULL;
        if (technique == SI_ORACLE_BITSET) {
            bits = (uint64_t*)malloc(nwords * sizeof(uint64_t));
            if (!bits) bad = 1;
        }
        for (uint32_t a = lower; a < upper && !bad; ++a) {
            if (technique == SI_ORACLE_BITSET) {
                bitset_row(elements, offsets, k, a, bits, nwords, counts);
                continue;
            }
            const uint32_t* sa = elements + offsets[a];
            uint64_t na = offsets[a + 1] - offsets[a];
            for (uint32_t b = a + 1; b < k; ++b) {
                const uint32_t* sb = elements + offsets[b];
                uint64_t nb = offsets[b + 1] - offsets[b];
                uint64_t c = technique == SI_ORACLE_STD
                                 ? si_oracle_set_intersection(sa, na, sb, nb, NULL)
                                 : si_oracle_serial_intersect(sa, na, sb, nb);
                counts[si_oracle_triangular_index(k, a, b)] = (uint32_t)c;
            }
        }
        free(bits);
    }
    return bad ? -1 : 0;
}

/* Counts for an explicit list of pairs (pairs[2p], pairs[2p+1]) -- the batched
 * query form; each pair is the std::set_intersection count of the two sets. */
int si_oracle_pairs(const uint32_t* elements, const uint64_t* offsets, uint32_t k,
                    const uint32_t* pairs, uint64_t npairs, int threads, uint32_t* counts)
{
#ifdef _OPENMP
    int T = threads > 0 ? threads : omp_get_max_threads();
#else
    (void)threads;
#endif
    int bad = 0;
#ifdef _OPENMP
#pragma omp parallel for num_threads(T) schedule(dynamic, 256) reduction(|:bad)
#endif
    for (int64_t p = 0; p < (int64_t)npairs; ++p) {
        uint32_t a = pairs[2 * p], b = pairs[2 * p + 1];
        if (a >= k || b >= k) { bad = 1; continue; }
        counts[p] = (uint32_t)si_oracle_set_intersection(
            elements + offsets[a], offsets[a + 1] - offsets[a],
            elements + offsets[b], offsets[b + 1] - offsets[b], NULL);
    }
    return bad ? -1 : 0;
}

/* 1 if x[0..n) is strictly increasing, else 0. */
int si_oracle_is_strictly_increasing(const uint32_t* x, uint64_t n)
{
    for (uint64_t i = 1; i < n; ++i)
        if (x[i - 1] >= x[i]) return 0;
    return 1;
}

/* ------------------------------------------------------------------------
 * Seeded inputs for the reference's CPU executables.
 *
 * si_oracle_gen_uniform: the same n-subset of [lo, hi) as the engine's
 * si_gen_uniform (so a reference run reads exactly the sets the engine was
 * timed on, without loading the engine's library).  Restated from its
 * definition:
 *   dense (n > U/64, U = hi - lo): the n values v with the smallest keys
 *     (hash32(seed, v) << 32 | (v - lo)), ascending; hash32 is the top half of
 *     the splitmix64 finaliser of v + seed * 0x9e3779b97f4a7c15 + 0x632be59bd9b4e019;
 *   sparse: the first n distinct values lo + floor(r * U / 2^64) of the
 *     splitmix64 stream that starts at seed * 0x9e3779b97f4a7c15 + 0x2545f4914f6cdd1d,
 *     sorted.
 * tests/test_oracle.py checks it against si_gen_uniform on both branches. */
static uint64_t gen_mix64(uint64_t x)
{
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    x ^= x >> 31;
    return x;
}

static uint32_t gen_hash32(uint64_t seed, uint64_t v)
{
    return (uint32_t)(gen_mix64(v + seed * 0x9e3779b97f4a7c15ull + 0x632be59bd9b4e019ull) >> 32);
}

static int cmp_u32(const void* x, const void* y)
{
    uint32_t a = *(const uint32_t*)x, b = *(const uint32_t*)y;
    return a < b ? -1 : a > b;
}

/* histogram of (hash >> 16), or of (hash & 0xffff) among hashes whose top half is bin1 */
static void gen_hist(uint64_t seed, uint64_t lo, uint64_t U, int level, uint64_t bin1, uint64_t* hist)
{
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
        uint64_t* h = calloc(65536, sizeof(uint64_t));
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int64_t v = 0; v < (int64_t)U; ++v) {
            uint32_t x = gen_hash32(seed, lo + (uint64_t)v);
            if (level == 0) ++h[x >> 16];
            else if ((x >> 16) == bin1) ++h[x & 0xffff];
        }
#ifdef _OPENMP
#pragma omp critical
#endif
        for (int q = 0; q < 65536; ++q) hist[q] += h[q];
        free(h);
    }
}

int si_oracle_gen_uniform(uint64_t seed, uint64_t n, uint64_t lo, uint64_t hi, uint32_t* out)
{
    if (hi < lo || hi - lo > (1ull << 32) || n > hi - lo) return -1;
    const uint64_t U = hi - lo;
    if (n == 0) return 0;
    if (n > U / 64) {
        /* threshold t = the n-th smallest hash; values with hash < t are all
         * taken, those with hash == t in increasing v until n are held */
        uint64_t* hist = calloc(65536, sizeof(uint64_t));
        if (!hist) return -2;
        gen_hist(seed, lo, U, 0, 0, hist);
        uint64_t need = n, bin1 = 0;
        for (; bin1 < 65536; ++bin1) {
            if (hist[bin1] >= need) break;
            need -= hist[bin1];
        }
        memset(hist, 0, 65536 * sizeof(uint64_t));
        gen_hist(seed, lo, U, 1, bin1, hist);
        uint64_t bin2 = 0;
        for (; bin2 < 65536; ++bin2) {
            if (hist[bin2] >= need) break;
            need -= hist[bin2];
        }
        free(hist);
        const uint32_t thr = (uint32_t)((bin1 << 16) | bin2);
        uint64_t p = 0, eq = 0;
        for (uint64_t v = 0; v < U; ++v) {
            uint32_t x = gen_hash32(seed, lo + v);
            if (x < thr || (x == thr && eq++ < need)) out[p++] = (uint32_t)(lo + v);
        }
        return p == n ? 0 : -3;
    }
    /* sparse: open-addressing set of the values drawn so far */
    uint64_t cap = 1;
    while (cap < 4 * n) cap <<= 1;
    uint64_t* table = calloc(cap, sizeof(uint64_t)); /* value + 1, 0 = empty */
    if (!table) return -2;
    uint64_t state = seed * 0x9e3779b97f4a7c15ull + 0x2545f4914f6cdd1dull, k = 0;
    while (k < n) {
        state += 0x9e3779b97f4a7c15ull;
        const uint64_t r = gen_mix64(state);
        const uint32_t v = (uint32_t)(lo + (uint64_t)(((unsigned __int128)r * U) >> 64));
        uint64_t s = gen_mix64(v) & (cap - 1);
        while (table[s] && table[s] != (uint64_t)v + 1) s = (s + 1) & (cap - 1);
        if (!table[s]) {
            table[s] = (uint64_t)v + 1;
            out[k++] = v;
        }
    }
    free(table);
    qsort(out, n, sizeof(uint32_t), cmp_u32);
    return 0;
}
