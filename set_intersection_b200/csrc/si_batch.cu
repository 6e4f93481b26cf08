// si_batch.cu -- counts of a batch of uneven pairs of one collection in one
// persistent launch.
//
// The reference has no batched mode: every pair is a host-loop iteration with
// its own launches (src/ip.cu:141-177 for one tile pair; a single pair costs
// the 3-kernel SISI path).  Here a list of (a, b) pairs of a CSR collection is
// counted by ONE persistent kernel:
//
//  * Work queue: the pairs are ordered by estimated cost, largest first (a
//    device radix sort of cost keys), and every warp takes the next pair from
//    an atomic ticket, so the long pairs start first and the short ones fill
//    the tail.
//  * Two techniques per pair, picked per bucket of (log2 of the smaller size,
//    log2 of the size ratio) from a 256-entry table:
//      MERGE (ip): the warp streams both sets through a shared-memory ring of
//        two 256-element blocks per set; every round finalises the elements up
//        to the smaller of the two window maxima, counts matches by binary
//        search of the A window's elements in the B window, and slides; the
//        next block of each set is prefetched into registers a round ahead.
//      SEARCH (obs): the warp takes the smaller set 256 elements at a time,
//        narrows the window of the larger set that can hold them (two binary
//        searches), then every lane runs 8 interleaved binary searches in it.
//  * The table comes from si_batch_tune, which times both techniques on a
//    sample of every populated bucket, or defaults to SEARCH when the larger
//    set is at least 16 times the smaller.
#include <algorithm>
#include <cstring>
#include <cub/device/device_radix_sort.cuh>
#include <vector>

#include "si_device.cuh"
#include "si_internal.h"

namespace si {
namespace {

constexpr int kBThreads = 256;            // 8 warps, 32 KiB of rings
constexpr int kBWarps = kBThreads / 32;
constexpr uint32_t kW = 256;             // window (block) per set per round
constexpr uint32_t kRing = 2 * kW;       // ring of two blocks per set
constexpr uint32_t kRingMask = kRing - 1;
constexpr int kVT = kW / 32;             // elements per lane per block
constexpr size_t kBatchHeader = 256;     // [0..16) error words, [16] u32 ticket
constexpr uint8_t kMerge = 0, kSearch = 1;

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

// Bucket of a pair: (log2 of the smaller size, log2 of larger / smaller), 4 bits each.
__host__ __device__ inline uint32_t pair_bucket(uint64_t na, uint64_t nb) {
    const uint64_t s = na < nb ? na : nb, l = na < nb ? nb : na;
    const uint32_t ls = s ? min(15u, log2_floor(s)) : 0u;
    const uint32_t lr = s ? min(15u, log2_floor(l / s)) : 15u;
    return (ls << 4) | lr;
}

struct TechTable {
    uint8_t t[256];
};

__device__ __forceinline__ uint64_t search_cost(uint64_t s, uint64_t l) {
    return s * (log2_floor(l + 1) + 4);
}

// Cost key per pair (descending cost, then pair index): the work queue order.
__global__ void batch_keys_kernel(const uint64_t* __restrict__ off, const uint32_t* __restrict__ pairs,
                                  uint64_t npairs, uint32_t k, TechTable table, int forced,
                                  uint64_t* __restrict__ keys, uint32_t* err) {
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < npairs; p += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t a = pairs[2 * p], b = pairs[2 * p + 1];
        uint64_t cost = 0;
        if (a >= k || b >= k) {
            record_error(err, SI_ERR_INVALID_INPUT, 50, static_cast<uint32_t>(p));
        } else {
            const uint64_t na = off[a + 1] - off[a], nb = off[b + 1] - off[b];
            const uint8_t t = forced >= 0 ? static_cast<uint8_t>(forced) : table.t[pair_bucket(na, nb)];
            cost = t == kSearch ? search_cost(min(na, nb), max(na, nb)) : na + nb;
        }
        const uint64_t c = min(cost, uint64_t(0xffffffffu));
        keys[p] = (uint64_t(0xffffffffu - c) << 32) | static_cast<uint32_t>(p);
    }
}

// ------------------------------------------------------ per-warp techniques --
__device__ __forceinline__ uint64_t lower_bound_g(const uint32_t* x, uint64_t lo, uint64_t hi, uint32_t v) {
    uint64_t len = hi - lo;
    while (len > 0) {
        const uint64_t half = len >> 1;
        const bool c = __ldg(x + lo + half) < v;
        lo = c ? lo + half + 1 : lo;
        len = c ? len - half - 1 : half;
    }
    return lo;
}

__device__ __forceinline__ uint64_t upper_bound_g(const uint32_t* x, uint64_t lo, uint64_t hi, uint32_t v) {
    uint64_t len = hi - lo;
    while (len > 0) {
        const uint64_t half = len >> 1;
        const bool c = __ldg(x + lo + half) <= v;
        lo = c ? lo + half + 1 : lo;
        len = c ? len - half - 1 : half;
    }
    return lo;
}

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

// Number of window elements w[0 .. len) (ring positions from i0) that are <= v.
__device__ __forceinline__ uint32_t ring_upper(const uint32_t* ring, uint64_t i0, uint32_t len, uint32_t v) {
    uint32_t lo = 0, n = len;
    while (n > 0) {
        const uint32_t half = n >> 1;
        const bool c = ring[(i0 + lo + half) & kRingMask] <= v;
        lo = c ? lo + half + 1 : lo;
        n = c ? n - half - 1 : half;
    }
    return lo;
}

// MERGE: |A ∩ B| by streaming both sets through the warp's rings.
__device__ uint32_t merge_pair(const uint32_t* A, uint64_t na, const uint32_t* B, uint64_t nb, uint32_t* ra,
                               uint32_t* rb, int lane) {
    if (na == 0 || nb == 0) return 0;
    if (__ldg(A + na - 1) < __ldg(B) || __ldg(B + nb - 1) < __ldg(A)) return 0;  // disjoint value ranges
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
        const uint32_t lastA = ra[(ia + la - 1) & kRingMask], lastB = rb[(ib + lb - 1) & kRingMask];
        const uint32_t m = min(lastA, lastB);
        // the elements of both windows up to m are final this round
        const uint32_t cA = lastA <= m ? la : ring_upper(ra, ia, la, m);
        const uint32_t cB = lastB <= m ? lb : ring_upper(rb, ib, lb, m);
#pragma unroll
        for (int t = 0; t < kVT; ++t) {
            const uint32_t j = lane + 32u * t;
            if (j < cA) {
                const uint32_t v = ra[(ia + j) & kRingMask];
                const uint32_t q = ring_upper(rb, ib, cB, v);  // elements <= v
                hits += (q > 0 && rb[(ib + q - 1) & kRingMask] == v) ? 1u : 0u;
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

// SEARCH: every element of the smaller set S, binary-searched in the larger L.
__device__ uint32_t search_pair(const uint32_t* S, uint64_t ns, const uint32_t* L, uint64_t nl, int lane) {
    if (ns == 0 || nl == 0) return 0;
    uint32_t hits = 0;
    uint64_t from = 0;  // the windows advance monotonically
    for (uint64_t base = 0; base < ns; base += kW) {
        const uint64_t last_i = min(base + kW, ns) - 1;
        // window of L that can hold S[base .. last_i]: lane 0 the lower end, lane 1 the upper
        uint64_t edge = 0;
        if (lane == 0) edge = lower_bound_g(L, from, nl, __ldg(S + base));
        if (lane == 1) edge = upper_bound_g(L, from, nl, __ldg(S + last_i));
        const uint64_t lo = __shfl_sync(kFullMask, edge, 0), hi = __shfl_sync(kFullMask, edge, 1);
        from = hi;
        if (lo >= hi) continue;
        uint32_t v[kVT];
        uint64_t pos[kVT], len[kVT];
#pragma unroll
        for (int t = 0; t < kVT; ++t) {
            const uint64_t i = base + lane + 32u * t;
            v[t] = i <= last_i ? __ldg(S + i) : 0u;
            pos[t] = lo;
            len[t] = i <= last_i ? hi - lo : 0;
        }
        // interleaved lower-bound searches: kVT independent load chains per lane
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
    return __reduce_add_sync(kFullMask, hits);
}

struct BatchParams {
    const uint32_t* el;
    const uint64_t* off;
    const uint32_t* pairs;
    uint64_t npairs;
    uint32_t k;
    const uint64_t* keys;  // sorted: low 32 bits = pair index (the queue order)
    const uint32_t* subset;  // when non-null: the queue is these pair indices, in order
    uint32_t* counts;
    uint32_t* ticket;
    int forced;            // -1: table; else kMerge / kSearch for every pair
    TechTable table;
};

__global__ void __launch_bounds__(kBThreads) batch_kernel(BatchParams p) {
    __shared__ __align__(16) uint32_t rings[kBWarps][2][kRing];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t* ra = rings[warp][0];
    uint32_t* rb = rings[warp][1];
    for (;;) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(p.ticket, 1u);
        t = __shfl_sync(kFullMask, t, 0);
        if (t >= p.npairs) break;
        const uint32_t pi = p.subset ? p.subset[t] : static_cast<uint32_t>(p.keys[t] & 0xffffffffu);
        const uint32_t a = p.pairs[2 * uint64_t(pi)], b = p.pairs[2 * uint64_t(pi) + 1];
        if (a >= p.k || b >= p.k) continue;  // recorded by the key kernel
        const uint64_t a0 = p.off[a], na = p.off[a + 1] - a0, b0 = p.off[b], nb = p.off[b + 1] - b0;
        const uint8_t tech = p.forced >= 0 ? static_cast<uint8_t>(p.forced) : p.table.t[pair_bucket(na, nb)];
        uint32_t c;
        if (tech == kSearch) {
            const bool as = na <= nb;
            c = search_pair(p.el + (as ? a0 : b0), as ? na : nb, p.el + (as ? b0 : a0), as ? nb : na, lane);
        } else {
            c = merge_pair(p.el + a0, na, p.el + b0, nb, ra, rb, lane);
        }
        if (lane == 0) p.counts[pi] = c;
        __syncwarp();
    }
}

TechTable default_table() {
    TechTable T;
    for (uint32_t b = 0; b < 256; ++b) T.t[b] = (b & 15u) >= 4 ? kSearch : kMerge;  // ratio >= 16: search
    return T;
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
    BatchParams prm;
    prm.el = d_elements;
    prm.off = d_offsets;
    prm.pairs = d_pairs;
    prm.npairs = d_subset ? nsubset : npairs;
    prm.k = k;
    prm.keys = keys;
    prm.subset = d_subset;
    prm.counts = d_counts;
    prm.ticket = reinterpret_cast<uint32_t*>(w + 16);
    prm.forced = forced;
    prm.table = table;
    if (!d_subset) {
        PhaseTimer timer("batch_plan", stream);
        const unsigned g = static_cast<unsigned>(std::min<uint64_t>((npairs + 255) / 256, uint64_t(sm_count()) * 8));
        batch_keys_kernel<<<g, 256, 0, stream>>>(d_offsets, d_pairs, npairs, k, table, forced, keys_in, err);
        SI_LAUNCH_CHECK("batch_keys_kernel");
        size_t tmp = L.cub_bytes;
        SI_CUDA_TRY(cub::DeviceRadixSort::SortKeys(w + L.off_cub, tmp, keys_in, keys, static_cast<int>(npairs), 0, 64,
                                                   stream));
    }
    int per_sm = 0;
    SI_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel, kBThreads, 0));
    const unsigned grid = static_cast<unsigned>(sm_count() * std::max(1, per_sm));
    PhaseTimer timer("batch_count", stream);
    batch_kernel<<<grid, kBThreads, 0, stream>>>(prm);
    SI_LAUNCH_CHECK("batch_kernel");
    return SI_OK;
}

__global__ void bucket_kernel(const uint64_t* __restrict__ off, const uint32_t* __restrict__ pairs, uint64_t npairs,
                              uint32_t k, uint8_t* __restrict__ bucket) {
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < npairs; p += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t a = pairs[2 * p], b = pairs[2 * p + 1];
        bucket[p] = (a < k && b < k) ? static_cast<uint8_t>(pair_bucket(off[a + 1] - off[a], off[b + 1] - off[b])) : 0;
    }
}

}  // namespace

size_t batch_workspace_size(uint64_t npairs) { return batch_layout(npairs).total; }

si_status batch_count(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, const uint32_t* d_pairs,
                      uint64_t npairs, si_technique t, const uint8_t* table, uint32_t* d_counts, void* ws,
                      size_t ws_bytes, cudaStream_t stream) {
    TechTable T = default_table();
    if (table) std::memcpy(T.t, table, 256);
    const int forced = t == SI_TECH_IP ? kMerge : t == SI_TECH_OBS ? kSearch : -1;
    return batch_launch(d_elements, d_offsets, k, d_pairs, npairs, T, forced, nullptr, 0, d_counts, ws, ws_bytes,
                        stream);
}

si_status batch_tune(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, const uint32_t* d_pairs,
                     uint64_t npairs, uint32_t sample, uint32_t* d_counts, void* ws, size_t ws_bytes,
                     cudaStream_t stream, uint8_t* table_out) {
    TechTable T = default_table();
    std::memcpy(table_out, T.t, 256);
    const BatchLayout L = batch_layout(npairs);
    if (ws_bytes < L.total) return SI_ERR_WORKSPACE_TOO_SMALL;
    if (npairs == 0) return SI_OK;
    // bucket of every pair, on the host
    unsigned char* w = static_cast<unsigned char*>(ws);
    uint8_t* d_bucket = reinterpret_cast<uint8_t*>(w + L.off_keys_in);  // scratch: npairs bytes
    const unsigned g = static_cast<unsigned>(std::min<uint64_t>((npairs + 255) / 256, uint64_t(sm_count()) * 8));
    bucket_kernel<<<g, 256, 0, stream>>>(d_offsets, d_pairs, npairs, k, d_bucket);
    SI_LAUNCH_CHECK("bucket_kernel");
    std::vector<uint8_t> bucket(npairs);
    SI_CUDA_TRY(cudaMemcpyAsync(bucket.data(), d_bucket, npairs, cudaMemcpyDeviceToHost, stream));
    SI_CUDA_TRY(cudaStreamSynchronize(stream));
    std::vector<std::vector<uint32_t>> members(256);
    for (uint64_t p = 0; p < npairs; ++p)
        if (members[bucket[p]].size() < sample) members[bucket[p]].push_back(static_cast<uint32_t>(p));
    // sample lists on the device, after the bucket bytes
    uint32_t* d_subset = reinterpret_cast<uint32_t*>(w + L.off_keys);  // npairs * 8 bytes of room
    cudaEvent_t e0, e1;
    SI_CUDA_TRY(cudaEventCreate(&e0));
    SI_CUDA_TRY(cudaEventCreate(&e1));
    si_status st = SI_OK;
    for (int b = 0; b < 256 && st == SI_OK; ++b) {
        const auto& m = members[b];
        if (m.size() < 32) continue;  // too few pairs to matter: keep the default
        if (cudaMemcpyAsync(d_subset, m.data(), m.size() * 4, cudaMemcpyHostToDevice, stream) != cudaSuccess) {
            st = cuda_fail(cudaGetLastError(), "batch_tune copy");
            break;
        }
        float ms[2] = {0, 0};
        for (int tech = 0; tech < 2 && st == SI_OK; ++tech) {
            for (int rep = 0; rep < 2 && st == SI_OK; ++rep) {  // the first run warms the caches
                cudaEventRecord(e0, stream);
                st = batch_launch(d_elements, d_offsets, k, d_pairs, npairs, T, tech, d_subset, m.size(), d_counts,
                                  ws, ws_bytes, stream);
                cudaEventRecord(e1, stream);
            }
            if (st != SI_OK) break;
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                st = cuda_fail(cudaGetLastError(), "batch_tune");
                break;
            }
            cudaEventElapsedTime(&ms[tech], e0, e1);
        }
        table_out[b] = ms[kSearch] < ms[kMerge] ? kSearch : kMerge;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}

}  // namespace si
