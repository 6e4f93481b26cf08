// si_batch.cu -- counts of a batch of uneven pairs of one collection in one
// persistent launch.
//
// The reference has no batched mode: every pair is a host-loop iteration with
// its own launches (src/ip.cu:141-177 for one tile pair; a single pair costs
// the 3-kernel SISI path).  Here a list of (a, b) pairs of a CSR collection is
// counted by two persistent kernels over one work queue:
//
//  * Work queue: the pairs are ordered by estimated cost, largest first (a
//    device radix sort of keys that carry each pair's technique), merge and
//    search pairs first, hash and bitmap pairs after them; every warp takes
//    the next pair of its kernel's part from an atomic ticket, so the long
//    pairs start first and the short ones fill the tail.  The merge / search
//    kernel runs 32 warps per SM (search is latency-bound), the hash / bitmap
//    kernel 24 with 8 KiB of shared memory each.
//  * Six technique codes per pair, picked per bucket of (density class of the
//    larger set, log2 of the smaller size, log2 of the size ratio) from a
//    1024-entry table:
//      MERGE (ip): the warp streams both sets through a shared-memory ring of
//        two 256-element blocks per set; every round finalises the elements up
//        to the smaller of the two window maxima and merges them along the
//        merge path (each lane an equal share of the merged positions after a
//        split search, as the reference's intersectPath splits a partition,
//        src/ip.cu:207-245), then slides; the next block of each set is
//        prefetched into registers a round ahead.
//      SEARCH (obs): the warp takes the smaller set 256 elements at a time,
//        bounds the window of the larger set that can hold them, caches 256
//        samples of a long window in shared memory, and every lane runs 8
//        interleaved binary searches in the gaps between samples.
//      HASH (hi, windows of 1024 or 512 elements): the smaller set S is cut
//        into windows of consecutive elements; each window goes into the
//        warp's 2048-slot open-addressing table (load <= 1/2 or 1/4) and the
//        elements of the larger set up to the window's last value probe it
//        (src/hi.cu:361-418 hashes one partition the same way).
//      BITMAP (windows of 16384 or 32768 values): both sets set bits in the
//        warp's two bitmaps of the window's values and the AND's popcount is
//        the window's count; the next window starts at the larger of the two
//        sets' next elements (src/bitmap_dynamic.cu:279-319 probes a set's
//        bitmap; this is the window form of si_sisi_bitmap.cu's engine).
//    HASH and BITMAP read both sets as 256-element streams (si_stream.cuh).
//  * The table comes from si_batch_tune, which times every technique on a
//    sample of every populated bucket, or the default rule.
#include <algorithm>
#include <cstring>
#include <cub/device/device_radix_sort.cuh>
#include <mutex>
#include <vector>

#include "si_device.cuh"
#include "si_internal.h"
#include "si_stream.cuh"

namespace si {
namespace {

constexpr int kBThreads = 256;           // 8 warps
constexpr int kBWarps = kBThreads / 32;
// Two kernels share the queue: the merge / search one (64 registers a thread,
// 32 KiB of rings: 4 CTAs, 32 warps per SM; search is latency-bound and wants
// the warps) and the stream one for hash and bitmap (80 registers, 8 KiB a
// warp: 3 CTAs, 24 warps per SM).
constexpr int kSearchCtasPerSm = 4;
constexpr int kStreamCtasPerSm = 3;
constexpr uint32_t kWarpSmem = 8192;     // stream kernel: shared bytes per warp, hash table or bitmaps
constexpr uint32_t kBSmem = kBWarps * kWarpSmem + 4096;  // + the skew to a 4 KiB boundary
constexpr uint32_t kW = 256;             // window (block) per set per round
constexpr uint32_t kRing = 2 * kW;       // ring of two blocks per set
constexpr uint32_t kRingMask = kRing - 1;
constexpr int kVT = kW / 32;             // elements per lane per block
// header: [0..16) error words, [16] u32 ticket of the merge / search kernel,
// [20] u32 ticket of the stream kernel, [24] u32 pairs in the merge / search
// part of the queue (its first part)
constexpr size_t kBatchHeader = 256;
// technique codes: the table's bytes (si.h SI_BATCH_*)
constexpr uint8_t kMerge = 0, kSearch = 1, kHash1024 = 2, kHash512 = 3, kBitmap16K = 4, kBitmap32K = 5;
constexpr uint8_t kTechCodes = 6;
constexpr uint32_t kTableSize = 1024;    // 4 density classes x 16 size classes x 16 ratio classes

struct BatchLayout {
    size_t off_keys_in = 0, off_keys = 0, off_cub = 0, cub_bytes = 0, total = 0;
};

BatchLayout batch_layout(uint64_t npairs) {
    BatchLayout L;
    size_t o = kBatchHeader;
    L.off_keys_in = o;  o = align_up(o + npairs * 8, 256);
    L.off_keys = o;     o = align_up(o + npairs * 8, 256);
    size_t sort_bytes = 0;
    if (cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, static_cast<const uint64_t*>(nullptr),
                                       static_cast<uint64_t*>(nullptr), static_cast<int>(std::max<uint64_t>(npairs, 1))) !=
        cudaSuccess)
        sort_bytes = npairs * 8 + (1u << 20);  // without a device to ask: a bound
    cudaGetLastError();
    L.cub_bytes = align_up(sort_bytes, 256);
    L.off_cub = o;
    o += L.cub_bytes;
    L.total = o;
    return L;
}

__host__ __device__ inline uint32_t log2_floor(uint64_t x) {  // x >= 1
#ifdef __CUDA_ARCH__
    return 63u - static_cast<uint32_t>(__clzll(static_cast<long long>(x)));
#else
    uint32_t r = 0;
    while (x >>= 1) ++r;
    return r;
#endif
}

// Density class of a set from its first and last values and size: the mean
// gap between consecutive values is < 4, < 32, < 256 or larger (class 0..3).
__host__ __device__ inline uint32_t density_class(uint32_t first, uint32_t last, uint64_t n) {
    if (n < 2) return 3;
    const uint64_t gap = static_cast<uint64_t>(last - first) / (n - 1);
    return gap < 4 ? 0u : gap < 32 ? 1u : gap < 256 ? 2u : 3u;
}

// Bucket of a pair: (density class of the larger set, log2 of the smaller
// size, log2 of larger / smaller): 2 + 4 + 4 bits.
__host__ __device__ inline uint32_t pair_bucket(uint64_t na, uint64_t nb, uint32_t dclass) {
    const uint64_t s = na < nb ? na : nb, l = na < nb ? nb : na;
    const uint32_t ls = s ? min(15u, log2_floor(s)) : 0u;
    const uint32_t lr = s ? min(15u, log2_floor(l / s)) : 15u;
    return (dclass << 8) | (ls << 4) | lr;
}

struct TechTable {
    uint8_t t[kTableSize];
};

__device__ __forceinline__ uint64_t search_cost(uint64_t s, uint64_t l) {
    return s * (log2_floor(l + 1) + 4);
}

struct PairSets {
    uint64_t a0, na, b0, nb;
};

__device__ __forceinline__ PairSets pair_sets(const uint64_t* off, uint32_t a, uint32_t b) {
    PairSets p;
    p.a0 = off[a];
    p.na = off[a + 1] - p.a0;
    p.b0 = off[b];
    p.nb = off[b + 1] - p.b0;
    return p;
}

// The pair's bucket: its larger set's density class comes from that set's end values.
__device__ __forceinline__ uint32_t device_bucket(const uint32_t* el, const PairSets& p) {
    const bool a_large = p.na >= p.nb;
    const uint64_t l0 = a_large ? p.a0 : p.b0, nl = a_large ? p.na : p.nb;
    const uint32_t dc = nl >= 2 ? density_class(__ldg(el + l0), __ldg(el + l0 + nl - 1), nl) : 3u;
    return pair_bucket(p.na, p.nb, dc);
}

__host__ __device__ constexpr bool is_stream_tech(uint8_t t) { return t >= kHash1024 && t < kTechCodes; }

// Queue key per pair: stream class (1 bit: hash or bitmap), descending cost
// (28 bits, saturated), technique (3 bits), pair index (32 bits).  Sorted
// ascending, the merge / search pairs come first, each part largest first;
// n_first counts the first part.  A stream technique falls back to merge for
// a pair whose larger set has 2^32 - 1024 elements or more (stream positions
// are 32-bit).
__global__ void batch_keys_kernel(const uint32_t* __restrict__ el, const uint64_t* __restrict__ off,
                                  const uint32_t* __restrict__ pairs, uint64_t npairs, uint32_t k, TechTable table,
                                  int forced, uint64_t* __restrict__ keys, uint32_t* err, uint32_t* n_first) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t end = (npairs + 31) / 32 * 32;  // whole warps, for the aggregated count
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < end; p += stride) {
        bool first_part = false;
        if (p < npairs) {
            const uint32_t a = pairs[2 * p], b = pairs[2 * p + 1];
            uint64_t cost = 0;
            uint8_t t = kMerge;
            if (a >= k || b >= k) {
                record_error(err, SI_ERR_INVALID_INPUT, 50, static_cast<uint32_t>(p));
            } else {
                const PairSets ps = pair_sets(off, a, b);
                t = forced >= 0 ? static_cast<uint8_t>(forced) : table.t[device_bucket(el, ps)];
                if (t >= kTechCodes || (is_stream_tech(t) && max(ps.na, ps.nb) >= kMaxStream)) t = kMerge;
                cost = t == kSearch ? search_cost(min(ps.na, ps.nb), max(ps.na, ps.nb)) : ps.na + ps.nb;
            }
            const uint64_t c = min(cost, uint64_t(0x0fffffffu));
            const uint64_t cls = is_stream_tech(t) ? 1u : 0u;
            keys[p] = (((cls << 28 | (0x0fffffffu - c)) << 3 | t) << 32) | static_cast<uint32_t>(p);
            first_part = cls == 0;
        }
        const uint32_t m = __ballot_sync(kFullMask, first_part);
        if ((threadIdx.x & 31) == 0 && m) atomicAdd(n_first, static_cast<uint32_t>(__popc(m)));
    }
}

// ------------------------------------------------------ per-warp techniques --
// Block `blk` of x (elements [blk*kW, blk*kW + kW) below n) into registers.
__device__ __forceinline__ void fetch_block(const uint32_t* x, uint64_t n, uint64_t blk, int lane, uint32_t (&r)[kVT]) {
    const uint64_t b0 = blk * kW;
#pragma unroll
    for (int t = 0; t < kVT; ++t) {
        const uint64_t i = b0 + lane + 32u * t;
        r[t] = i < n ? __ldg(x + i) : 0u;
    }
}

__device__ __forceinline__ void store_block(uint32_t* ring, uint64_t blk, int lane, const uint32_t (&r)[kVT]) {
    const uint32_t s0 = static_cast<uint32_t>((blk * kW) & kRingMask);
#pragma unroll
    for (int t = 0; t < kVT; ++t) ring[s0 + lane + 32u * t] = r[t];
}

// Number of window elements w[0 .. len) (ring positions from o) that are <= v,
// warp-cooperative, for a sorted window of len <= 256: lane l
// tests element 8 l, then the first eight lanes the elements of the one group
// of eight the answer ends in (two shared loads and two ballots per lane).
// Every lane gets the result.
__device__ __forceinline__ uint32_t ring_count_le(const uint32_t* ring, uint32_t o, uint32_t len, uint32_t v,
                                                  uint32_t lane) {
    const uint32_t i1 = 8 * lane;
    const uint32_t k = __popc(__ballot_sync(kFullMask, i1 < len && ring[(o + i1) & kRingMask] <= v));
    if (k == 0) return 0;
    const uint32_t i2 = 8 * (k - 1) + (lane & 7);
    const bool c2 = lane < 8 && i2 < len && ring[(o + i2) & kRingMask] <= v;
    return 8 * (k - 1) + __popc(__ballot_sync(kFullMask, c2));
}

// MERGE: |A ∩ B| by streaming both sets through the warp's rings: A's at
// ring[0, kRing), B's at ring[kRing, 2 kRing).  Ring offsets are 32-bit.
__device__ uint32_t merge_pair(const uint32_t* A, uint64_t na, const uint32_t* B, uint64_t nb, uint32_t* ring,
                               int lane) {
    if (na == 0 || nb == 0) return 0;
    if (__ldg(A + na - 1) < __ldg(B) || __ldg(B + nb - 1) < __ldg(A)) return 0;  // disjoint value ranges
    uint32_t* ra = ring;
    uint32_t* rb = ring + kRing;
    uint32_t pa[kVT], pb[kVT];
    // blocks 0 and 1 of each set into the rings, block 2 into registers
    fetch_block(A, na, 0, lane, pa);
    store_block(ra, 0, lane, pa);
    fetch_block(B, nb, 0, lane, pb);
    store_block(rb, 0, lane, pb);
    fetch_block(A, na, 1, lane, pa);
    store_block(ra, 1, lane, pa);
    fetch_block(B, nb, 1, lane, pb);
    store_block(rb, 1, lane, pb);
    fetch_block(A, na, 2, lane, pa);
    fetch_block(B, nb, 2, lane, pb);

    uint64_t ia = 0, ib = 0, LA = 0, LB = 0;  // LA: first element of the ring's older block
    uint32_t hits = 0;
    __syncwarp();
    for (;;) {
        const uint32_t la = na - ia < kW ? static_cast<uint32_t>(na - ia) : kW;
        const uint32_t lb = nb - ib < kW ? static_cast<uint32_t>(nb - ib) : kW;
        if (la == 0 || lb == 0) break;
        const uint32_t oa = static_cast<uint32_t>(ia) & kRingMask, ob = static_cast<uint32_t>(ib) & kRingMask;
        const uint32_t lastA = ra[(oa + la - 1) & kRingMask], lastB = rb[(ob + lb - 1) & kRingMask];
        const uint32_t m = min(lastA, lastB);
        // the elements of both windows up to m are final this round
        const uint32_t cA = lastA <= m ? la : ring_count_le(ra, oa, la, m, lane);
        const uint32_t cB = lastB <= m ? lb : ring_count_le(rb, ob, lb, m, lane);
        // merge path over the round's cA + cB (<= 512) final elements: lane l
        // takes merged positions [st l, st l + st), st = ceil(total / 32) (a
        // warp-uniform trip count, so no lane idles on short rounds); ties take
        // the A element first, and an A element equal to the B element after
        // it is a match
        {
            const uint32_t tot = cA + cB;
            const uint32_t st = (tot + 31) / 32;
            const uint32_t d = min(st * lane, tot), dend = min(d + st, tot);
            // a = A elements among the first d merged: the first a in
            // [max(0, d - cB), min(d, cA)] with A[a] > B[d - 1 - a]
            uint32_t lo = d > cB ? d - cB : 0u, hi = min(d, cA);
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                const bool right = ra[(oa + mid) & kRingMask] <= rb[(ob + d - 1 - mid) & kRingMask];
                lo = right ? mid + 1 : lo;
                hi = right ? hi : mid;
            }
            uint32_t a = lo, b = d - lo;
            uint32_t va = ra[(oa + a) & kRingMask], vb = rb[(ob + b) & kRingMask];
            // branch-free steps; a value read past cA or cB is never used
#pragma unroll 4
            for (uint32_t x = 0; x < st; ++x) {
                if (d + x < dend) {
                    const bool aok = a < cA, bok = b < cB;
                    const bool takeA = aok && (!bok || va <= vb);
                    hits += (takeA && bok && va == vb) ? 1u : 0u;
                    a += takeA ? 1u : 0u;
                    b += takeA ? 0u : 1u;
                    const uint32_t v = ring[takeA ? ((oa + a) & kRingMask) : (kRing + ((ob + b) & kRingMask))];
                    va = takeA ? v : va;
                    vb = takeA ? vb : v;
                }
            }
        }
        ia += cA;
        ib += cB;
        __syncwarp();
        // slide a ring whose older block is consumed: the prefetched block
        // takes its slot and the next one is fetched
        if (ia > LA + kW) {
            store_block(ra, LA / kW + 2, lane, pa);
            LA += kW;
            fetch_block(A, na, LA / kW + 2, lane, pa);
        }
        if (ib > LB + kW) {
            store_block(rb, LB / kW + 2, lane, pb);
            LB += kW;
            fetch_block(B, nb, LB / kW + 2, lane, pb);
        }
        __syncwarp();
    }
    return __reduce_add_sync(kFullMask, hits);
}

// SEARCH: every element of the smaller set S, binary-searched in the larger
// L, 256 elements of S at a time.  The window of L that can hold the block
// comes from two 32-ary warp searches; a window longer than 512 elements is
// sampled at 256 evenly spaced positions into shared memory (one load round
// for the warp, the cached top of the search tree, as the reference's obs
// caches it, src/obs.cu:275-438), every element finds its gap between two
// samples there, and only the gap is searched in global memory, 8 searches
// interleaved per lane.  samp: the warp's 256 words of shared memory.
constexpr uint32_t kSample = 256;
__device__ uint32_t search_pair(const uint32_t* S, uint64_t ns, const uint32_t* L, uint64_t nl, uint32_t* samp,
                               int lane) {
    if (ns == 0 || nl == 0) return 0;
    uint32_t hits = 0;
    uint64_t from = 0;  // the windows advance monotonically
    for (uint64_t base = 0; base < ns; base += kW) {
        const uint64_t last_i = min(base + kW, ns) - 1;
        // a smaller set of one block searches all of L (its samples bound the
        // gaps as well as a narrowed window would, without the two searches)
        // later blocks start where the previous one's window ended (the L
        // elements between are below this block's first value: harmless)
        uint64_t lo = 0, hi = nl;
        if (ns > kW) {
            const uint32_t v1 = __ldg(S + last_i);
            if (base == 0) {
                const uint32_t v0 = __ldg(S);
                lo = warp_first_true(0, nl, [&](uint64_t i) { return __ldg(L + i) >= v0; });
            } else {
                lo = from;
            }
            hi = warp_first_true(lo, nl, [&](uint64_t i) { return __ldg(L + i) > v1; });
        }
        from = hi;
        if (lo >= hi) continue;
        const uint64_t W = hi - lo;
        const bool sampled = W > 2 * kSample;
        if (sampled) {
#pragma unroll
            for (uint32_t t = 0; t < kSample / 32; ++t) {
                const uint32_t j = lane + 32 * t;
                samp[j] = __ldg(L + lo + W * j / kSample);
            }
            __syncwarp();
        }
        uint32_t v[kVT];
        uint64_t pos[kVT], len[kVT];
#pragma unroll
        for (int t = 0; t < kVT; ++t) {
            const uint64_t i = base + lane + 32u * t;
            v[t] = i <= last_i ? __ldg(S + i) : 0u;
            pos[t] = lo;
            len[t] = i <= last_i ? W : 0;
        }
        if (sampled) {
#pragma unroll
            for (int t = 0; t < kVT; ++t) {
                // c = samples <= v; the answer lies between samples c - 1 and c
                uint32_t c = 0;
#pragma unroll
                for (uint32_t step = kSample / 2; step > 0; step >>= 1)
                    c = samp[c + step - 1] <= v[t] ? c + step : c;
                c = (c == kSample - 1 && samp[kSample - 1] <= v[t]) ? kSample : c;
                const uint64_t p0 = lo + W * (c ? c - 1 : 0) / kSample;
                const uint64_t p1 = c == kSample ? hi : lo + W * c / kSample;
                pos[t] = p0;
                len[t] = c == 0 ? 0 : (len[t] ? p1 - p0 : 0);  // c == 0: v is below L[lo]
            }
            __syncwarp();  // the samples are read before the next block writes them
        }
        // interleaved searches for the last element <= v: kVT independent load
        // chains per lane, in 32-bit offsets from lo when the window allows
        if (W < (uint64_t(1) << 32)) {
            const uint32_t* Lw = L + lo;
            uint32_t o32[kVT], n32[kVT];
#pragma unroll
            for (int t = 0; t < kVT; ++t) {
                o32[t] = static_cast<uint32_t>(pos[t] - lo);
                n32[t] = static_cast<uint32_t>(len[t]);
            }
            // 4-ary steps (three independent loads, a quarter of the gap
            // left) while the gap allows, then binary: half the dependent
            // load rounds of a binary search
            bool more = true;
            while (more) {
                more = false;
#pragma unroll
                for (int t = 0; t < kVT; ++t) {
                    const uint32_t n = n32[t];
                    if (n >= 4) {
                        const uint32_t q1 = n >> 2, q2 = n >> 1, q3 = q1 + q2;
                        const uint32_t o = o32[t];
                        const bool c1 = __ldg(Lw + o + q1) <= v[t];
                        const bool c2 = __ldg(Lw + o + q2) <= v[t];
                        const bool c3 = __ldg(Lw + o + q3) <= v[t];
                        const uint32_t lo_q = c3 ? q3 : c2 ? q2 : c1 ? q1 : 0u;
                        const uint32_t hi_q = c3 ? n : c2 ? q3 : c1 ? q2 : q1;
                        o32[t] = o + lo_q;
                        n32[t] = hi_q - lo_q;
                        more |= n32[t] > 1;
                    } else if (n > 1) {
                        const uint32_t half = n >> 1;
                        const bool c = __ldg(Lw + o32[t] + half) <= v[t];
                        o32[t] = c ? o32[t] + half : o32[t];
                        n32[t] = c ? n - half : half;
                        more |= n32[t] > 1;
                    }
                }
            }
#pragma unroll
            for (int t = 0; t < kVT; ++t) hits += (n32[t] == 1 && __ldg(Lw + o32[t]) == v[t]) ? 1u : 0u;
        } else {
            bool more = true;
            while (more) {
                more = false;
#pragma unroll
                for (int t = 0; t < kVT; ++t) {
                    if (len[t] > 1) {
                        const uint64_t half = len[t] >> 1;
                        const bool c = __ldg(L + pos[t] + half) <= v[t];
                        pos[t] = c ? pos[t] + half : pos[t];
                        len[t] = c ? len[t] - half : half;
                        more |= len[t] > 1;
                    }
                }
            }
#pragma unroll
            for (int t = 0; t < kVT; ++t) hits += (len[t] == 1 && __ldg(L + pos[t]) == v[t]) ? 1u : 0u;
        }
    }
    return __reduce_add_sync(kFullMask, hits);
}

// ---------------------------------------------------------------- HASH --
// HASH: |S ∩ L| (S the smaller set), windows of kWinChunks chunks of S.
template <uint32_t kWinChunks>
__device__ uint32_t hash_pair(const uint32_t* S, uint64_t ns, const uint32_t* L, uint64_t nl, uint32_t* tab,
                              uint32_t lane) {
    static_assert(kWinChunks * kChunk <= kWinHashSlots / 2, "a window fills at most half of the table");
    if (ns == 0 || nl == 0) return 0;
    // the value 2^32 - 1 marks empty slots: a match of it is counted here and
    // it leaves both sets (it can only be their last element)
    const bool s_top = __ldg(S + ns - 1) == kWinHashEmpty, l_top = __ldg(L + nl - 1) == kWinHashEmpty;
    const uint32_t extra = s_top && l_top ? 1u : 0u;
    ns -= s_top;
    nl -= l_top;
    if (ns == 0 || nl == 0) return extra;
    const uint32_t lo = max(__ldg(S), __ldg(L));
    if (__ldg(S + ns - 1) < lo || __ldg(L + nl - 1) < lo) return extra;  // value ranges apart
    const uint64_t s0 = warp_first_true(0, ns, [&](uint64_t i) { return __ldg(S + i) >= lo; });
    const uint64_t l0 = warp_first_true(0, nl, [&](uint64_t i) { return __ldg(L + i) >= lo; });
    SetStream ss, sl;
    stream_init(ss, S, s0, ns, lane);
    stream_init(sl, L, l0, nl, lane);
    const uint32_t lv0 = sl.v1 - static_cast<uint32_t>(nl - l0);  // L's first stream position
    uint4* tab4 = reinterpret_cast<uint4*>(tab);
    uint32_t hits = 0;
    for (;;) {
        for (uint32_t i = lane; i < kWinHashSlots / 4; i += 32)
            tab4[i] = make_uint4(kWinHashEmpty, kWinHashEmpty, kWinHashEmpty, kWinHashEmpty);
        __syncwarp();
        // the window: the next kWinChunks chunks of S, up to its last value hi
        uint32_t hi = 0;
        bool more_s = true;
        for (uint32_t c = 0; c < kWinChunks && more_s; ++c) {
            if (ss.ph == 0)
                chunk_hash_insert(tab, ss.a0, ss.a1);
            else
                chunk_hash_insert(tab, ss.b0, ss.b1);
            hi = ss.last;
            more_s = stream_next(ss, lane);
        }
        __syncwarp();
        // L's elements up to hi probe it; a chunk reaching past hi stays
        bool more_l = true;
        for (;;) {
            if (sl.ph == 0)
                hits += __popc(chunk_hash_probe(tab, sl.a0, sl.a1, probe_mask(sl, sl.a0, sl.a1, lv0, hi, lane)));
            else
                hits += __popc(chunk_hash_probe(tab, sl.b0, sl.b1, probe_mask(sl, sl.b0, sl.b1, lv0, hi, lane)));
            if (sl.last > hi) break;
            more_l = stream_next(sl, lane);
            if (!more_l) break;
        }
        if (!more_l || !more_s) break;
        __syncwarp();  // the probes are done before the table is cleared
    }
    return __reduce_add_sync(kFullMask, hits) + extra;
}

// -------------------------------------------------------------- BITMAP --
// BITMAP: |X ∩ Y| by windows of 32 kWords values; bmx: the warp's two
// kWords-word bitmaps (bmx, bmx + kWords), each aligned to its size.
template <uint32_t kWords>
__device__ uint32_t bitmap_pair(const uint32_t* X, uint64_t nx, const uint32_t* Y, uint64_t ny, uint32_t* bmx,
                                uint32_t lane) {
    constexpr uint32_t kWinV = 32 * kWords;
    if (nx == 0 || ny == 0) return 0;
    const uint32_t lo = max(__ldg(X), __ldg(Y));
    if (__ldg(X + nx - 1) < lo || __ldg(Y + ny - 1) < lo) return 0;  // value ranges apart
    uint4* bx4 = reinterpret_cast<uint4*>(bmx);
    uint4* by4 = reinterpret_cast<uint4*>(bmx + kWords);
    for (uint32_t i = lane; i < kWords / 2; i += 32) bx4[i] = make_uint4(0u, 0u, 0u, 0u);  // both bitmaps
    const uint64_t x0 = warp_first_true(0, nx, [&](uint64_t i) { return __ldg(X + i) >= lo; });
    const uint64_t y0 = warp_first_true(0, ny, [&](uint64_t i) { return __ldg(Y + i) >= lo; });
    SetStream sx, sy;
    stream_init(sx, X, x0, nx, lane);
    stream_init(sy, Y, y0, ny, lane);
    const uint32_t sbx = smem_addr(bmx), sby = smem_addr(bmx + kWords);
    uint32_t a = max(__ldg(X + x0), __ldg(Y + y0));
    uint32_t hits = 0;
    __syncwarp();
    for (;;) {
        const uint64_t e = static_cast<uint64_t>(a) + kWinV;
        const uint32_t lim = e > 0xffffffffull ? static_cast<uint32_t>(0x100000000ull - a) : kWinV;
        const bool more_x = stream_fill<kWords>(sx, sbx, a, lim, e, lane);
        const bool more_y = stream_fill<kWords>(sy, sby, a, lim, e, lane);
        __syncwarp();
#pragma unroll
        for (uint32_t h = 0; h < kWords / 128; ++h) {
            const uint32_t i = 32 * h + lane;
            const uint4 p = bx4[i], q = by4[i];
            bx4[i] = make_uint4(0u, 0u, 0u, 0u);
            by4[i] = make_uint4(0u, 0u, 0u, 0u);
            hits += __popc(p.x & q.x) + __popc(p.y & q.y) + __popc(p.z & q.z) + __popc(p.w & q.w);
        }
        __syncwarp();
        if (!more_x || !more_y) break;
        a = max(stream_first_from(sx, e), stream_first_from(sy, e));
    }
    return __reduce_add_sync(kFullMask, hits);
}

// --------------------------------------------------------------- kernel --
struct BatchParams {
    const uint32_t* el;
    const uint64_t* off;
    const uint32_t* pairs;
    uint32_t k;
    const uint64_t* keys;    // sorted queue keys: technique in bits 32..34, pair index in the low 32
    const uint32_t* subset;  // when non-null: the queue is these pair indices, in order, all by `forced`
    uint64_t nqueue;         // queue length (all pairs, or the subset)
    const uint32_t* n_first; // pairs in the queue's first part (merge / search), from the key kernel
    uint32_t* counts;
    uint32_t* ticket;        // this kernel's ticket
    int forced;
};

// One kernel per part of the queue.  kStream = false: merge and search pairs
// (the first part), rings in static shared memory; kStream = true: hash and
// bitmap pairs (the rest), 8 KiB of dynamic shared memory per warp.  With a
// subset (the tuner) the kernel of the forced technique takes it all.
template <bool kStream>
__global__ void __launch_bounds__(kBThreads, kStream ? kStreamCtasPerSm : kSearchCtasPerSm)
    batch_kernel(BatchParams p) {
    extern __shared__ __align__(16) uint32_t smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // stream kernel: the warp's 8 KiB, 4 KiB aligned (the bitmaps' word
    // addresses are one LOP3); merge / search kernel: the warp's two rings
    uint32_t* region;
    if constexpr (kStream) {
        const uint32_t skew = ((smem_addr(smem) + 4095u) & ~4095u) - smem_addr(smem);
        region = smem + skew / 4 + warp * (kWarpSmem / 4);
    } else {
        __shared__ __align__(16) uint32_t rings[kBWarps][2 * kRing];
        region = rings[warp];
    }
    uint64_t q0 = 0, q1 = p.nqueue;
    if (!p.subset) {
        const uint32_t nf = *p.n_first;
        q0 = kStream ? nf : 0;
        q1 = kStream ? p.nqueue : nf;
    }
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(p.ticket, 1u);
        const uint64_t q = q0 + __shfl_sync(kFullMask, t, 0);
        if (q >= q1) break;
        uint32_t pi;
        uint8_t tech;
        if (p.subset) {
            pi = p.subset[q];
            tech = static_cast<uint8_t>(p.forced);
        } else {
            const uint64_t key = p.keys[q];
            pi = static_cast<uint32_t>(key);
            tech = static_cast<uint8_t>((key >> 32) & 7u);
        }
        const uint32_t a = p.pairs[2 * uint64_t(pi)], b = p.pairs[2 * uint64_t(pi) + 1];
        if (a >= p.k || b >= p.k) continue;  // recorded by the key kernel
        const PairSets ps = pair_sets(p.off, a, b);
        const bool as = ps.na <= ps.nb;  // A is the smaller set
        const uint32_t* S = p.el + (as ? ps.a0 : ps.b0);
        const uint32_t* L = p.el + (as ? ps.b0 : ps.a0);
        const uint64_t ns = as ? ps.na : ps.nb, nl = as ? ps.nb : ps.na;
        uint32_t c;
        if constexpr (kStream) {
            if (nl >= kMaxStream) tech = kMerge;  // only reachable with a tuner subset
            switch (tech) {
                case kMerge:
                    c = merge_pair(p.el + ps.a0, ps.na, p.el + ps.b0, ps.nb, region, lane);
                    break;
                case kHash512: c = hash_pair<2>(S, ns, L, nl, region, lane); break;
                case kBitmap16K: c = bitmap_pair<512>(L, nl, S, ns, region, lane); break;
                case kBitmap32K: c = bitmap_pair<1024>(L, nl, S, ns, region, lane); break;
                default: c = hash_pair<4>(S, ns, L, nl, region, lane); break;
            }
        } else {
            if (tech == kSearch)
                c = search_pair(S, ns, L, nl, region, lane);
            else
                c = merge_pair(p.el + ps.a0, ps.na, p.el + ps.b0, ps.nb, region, lane);
        }
        if (lane == 0) p.counts[pi] = c;
        __syncwarp();
    }
}

// Default rule: search when the larger set is at least 16 times the smaller,
// else hash.
TechTable default_table() {
    TechTable T;
    for (uint32_t b = 0; b < kTableSize; ++b) T.t[b] = (b & 15u) >= 4 ? kSearch : kHash1024;
    return T;
}

// Resident CTAs per SM of the two batch kernels on the current device (the
// stream kernel's shared-memory attribute is set per device, once).
struct BatchOccupancy {
    int search = 0, stream = 0;
};
BatchOccupancy batch_occupancy() {
    constexpr int kMaxDevices = 64;
    static BatchOccupancy cached[kMaxDevices];
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return {};
    std::lock_guard<std::mutex> lk(mu);
    BatchOccupancy& o = cached[dev];
    if (o.search == 0 || o.stream == 0) {
        int a = 0, b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, batch_kernel<false>, kBThreads, 0) != cudaSuccess ||
            cudaFuncSetAttribute(batch_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBSmem) !=
                cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, batch_kernel<true>, kBThreads, kBSmem) != cudaSuccess)
            return {};
        o.search = a;
        o.stream = b;
    }
    return o;
}

si_status batch_launch(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, const uint32_t* d_pairs,
                       uint64_t npairs, const TechTable& table, int forced, const uint32_t* d_subset,
                       uint64_t nsubset, uint32_t* d_counts, void* ws, size_t ws_bytes, cudaStream_t stream) {
    const BatchLayout L = batch_layout(npairs);
    if (ws_bytes < L.total) return SI_ERR_WORKSPACE_TOO_SMALL;
    unsigned char* w = static_cast<unsigned char*>(ws);
    uint32_t* err = reinterpret_cast<uint32_t*>(w);
    SI_CUDA_TRY(cudaMemsetAsync(w, 0, kBatchHeader, stream));
    if (npairs == 0) return SI_OK;
    uint64_t* keys_in = reinterpret_cast<uint64_t*>(w + L.off_keys_in);
    uint64_t* keys = reinterpret_cast<uint64_t*>(w + L.off_keys);
    uint32_t* n_first = reinterpret_cast<uint32_t*>(w + 24);
    BatchParams prm;
    prm.el = d_elements;
    prm.off = d_offsets;
    prm.pairs = d_pairs;
    prm.k = k;
    prm.keys = keys;
    prm.subset = d_subset;
    prm.nqueue = d_subset ? nsubset : npairs;
    prm.n_first = n_first;
    prm.counts = d_counts;
    prm.forced = forced;
    if (!d_subset) {
        PhaseTimer timer("batch_plan", stream);
        const unsigned g = static_cast<unsigned>(std::min<uint64_t>((npairs + 255) / 256, uint64_t(sm_count()) * 8));
        batch_keys_kernel<<<g, 256, 0, stream>>>(d_elements, d_offsets, d_pairs, npairs, k, table, forced, keys_in,
                                                 err, n_first);
        SI_LAUNCH_CHECK("batch_keys_kernel");
        size_t tmp = L.cub_bytes;
        SI_CUDA_TRY(cub::DeviceRadixSort::SortKeys(w + L.off_cub, tmp, keys_in, keys, static_cast<int>(npairs), 0, 64,
                                                   stream));
    }
    const BatchOccupancy occ = batch_occupancy();
    const int search_per_sm = occ.search, stream_per_sm = occ.stream;
    if (search_per_sm == 0 || stream_per_sm == 0) return cuda_fail(cudaGetLastError(), "batch_kernel attributes");
    // the subset of the tuner runs in its technique's kernel; the whole queue
    // in both, one part each (no stream part when every pair merges or searches)
    const bool forced_stream = forced >= 0 && is_stream_tech(static_cast<uint8_t>(forced));
    const bool run_search = d_subset ? !forced_stream : true;
    const bool run_stream = d_subset ? forced_stream : forced < 0 || forced_stream;
    PhaseTimer timer("batch_count", stream);
    if (run_search) {
        prm.ticket = reinterpret_cast<uint32_t*>(w + 16);
        batch_kernel<false><<<static_cast<unsigned>(sm_count() * search_per_sm), kBThreads, 0, stream>>>(prm);
        SI_LAUNCH_CHECK("batch_kernel<merge/search>");
    }
    if (run_stream) {
        prm.ticket = reinterpret_cast<uint32_t*>(w + 20);
        batch_kernel<true><<<static_cast<unsigned>(sm_count() * stream_per_sm), kBThreads, kBSmem, stream>>>(prm);
        SI_LAUNCH_CHECK("batch_kernel<hash/bitmap>");
    }
    return SI_OK;
}

__global__ void bucket_kernel(const uint32_t* __restrict__ el, const uint64_t* __restrict__ off,
                              const uint32_t* __restrict__ pairs, uint64_t npairs, uint32_t k,
                              uint16_t* __restrict__ bucket) {
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < npairs; p += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t a = pairs[2 * p], b = pairs[2 * p + 1];
        bucket[p] = (a < k && b < k) ? static_cast<uint16_t>(device_bucket(el, pair_sets(off, a, b))) : 0;
    }
}

}  // namespace

size_t batch_workspace_size(uint64_t npairs) { return batch_layout(npairs).total; }

si_status batch_count(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, const uint32_t* d_pairs,
                      uint64_t npairs, si_technique t, const uint8_t* table, uint32_t* d_counts, void* ws,
                      size_t ws_bytes, cudaStream_t stream) {
    TechTable T = default_table();
    if (table) std::memcpy(T.t, table, kTableSize);
    const int forced = t == SI_TECH_IP       ? kMerge
                       : t == SI_TECH_OBS    ? kSearch
                       : t == SI_TECH_HI     ? kHash1024
                       : t == SI_TECH_BITMAP ? kBitmap16K
                                             : -1;
    return batch_launch(d_elements, d_offsets, k, d_pairs, npairs, T, forced, nullptr, 0, d_counts, ws, ws_bytes,
                        stream);
}

si_status batch_tune(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, const uint32_t* d_pairs,
                     uint64_t npairs, uint32_t sample, uint32_t* d_counts, void* ws, size_t ws_bytes,
                     cudaStream_t stream, uint8_t* table_out) {
    TechTable T = default_table();
    std::memcpy(table_out, T.t, kTableSize);
    const BatchLayout L = batch_layout(npairs);
    if (ws_bytes < L.total) return SI_ERR_WORKSPACE_TOO_SMALL;
    if (npairs == 0) return SI_OK;
    // bucket of every pair, on the device, read back
    unsigned char* w = static_cast<unsigned char*>(ws);
    uint16_t* d_bucket = reinterpret_cast<uint16_t*>(w + L.off_keys_in);  // scratch: 2 npairs bytes
    const unsigned g = static_cast<unsigned>(std::min<uint64_t>((npairs + 255) / 256, uint64_t(sm_count()) * 8));
    bucket_kernel<<<g, 256, 0, stream>>>(d_elements, d_offsets, d_pairs, npairs, k, d_bucket);
    SI_LAUNCH_CHECK("bucket_kernel");
    std::vector<uint16_t> bucket(npairs);
    SI_CUDA_TRY(cudaMemcpyAsync(bucket.data(), d_bucket, npairs * 2, cudaMemcpyDeviceToHost, stream));
    SI_CUDA_TRY(cudaStreamSynchronize(stream));
    std::vector<std::vector<uint32_t>> members(kTableSize);
    for (uint64_t p = 0; p < npairs; ++p)
        if (members[bucket[p]].size() < sample) members[bucket[p]].push_back(static_cast<uint32_t>(p));
    // sample lists on the device, in the queue keys' room
    uint32_t* d_subset = reinterpret_cast<uint32_t*>(w + L.off_keys);  // npairs * 8 bytes of room
    cudaEvent_t e0, e1;
    SI_CUDA_TRY(cudaEventCreate(&e0));
    SI_CUDA_TRY(cudaEventCreate(&e1));
    si_status st = SI_OK;
    for (uint32_t b = 0; b < kTableSize && st == SI_OK; ++b) {
        const auto& m = members[b];
        if (m.size() < 32) continue;  // too few pairs to matter: keep the default
        if (cudaMemcpyAsync(d_subset, m.data(), m.size() * 4, cudaMemcpyHostToDevice, stream) != cudaSuccess) {
            st = cuda_fail(cudaGetLastError(), "batch_tune copy");
            break;
        }
        float ms[kTechCodes] = {};
        for (uint8_t tech = 0; tech < kTechCodes && st == SI_OK; ++tech) {
            // three runs: the first warms the caches, the faster of the other two counts
            ms[tech] = 0.f;
            for (int rep = 0; rep < 3 && st == SI_OK; ++rep) {
                cudaEventRecord(e0, stream);
                st = batch_launch(d_elements, d_offsets, k, d_pairs, npairs, T, tech, d_subset, m.size(), d_counts,
                                  ws, ws_bytes, stream);
                cudaEventRecord(e1, stream);
                if (st != SI_OK || rep == 0) continue;
                if (cudaEventSynchronize(e1) != cudaSuccess) {
                    st = cuda_fail(cudaGetLastError(), "batch_tune");
                    break;
                }
                float t = 0.f;
                cudaEventElapsedTime(&t, e0, e1);
                ms[tech] = rep == 1 ? t : std::min(ms[tech], t);
            }
            if (st != SI_OK) break;
        }
        if (st != SI_OK) break;
        // another technique replaces the default only when it is 3 % faster
        uint8_t best = T.t[b];
        for (uint8_t tech = 0; tech < kTechCodes; ++tech)
            if (ms[tech] < 0.97f * ms[best]) best = tech;
        table_out[b] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}

}  // namespace si
