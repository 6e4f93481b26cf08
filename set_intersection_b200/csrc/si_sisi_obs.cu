// si_sisi_obs.cu -- optimized binary search (obs) for one pair of sorted sets.
//
// The reference's obs (src/obs.cu:275-358, warpBasedOBS; :439-522 for the
// single pair) caches the first levels of the larger set's binary-search tree
// in shared memory and lets every element of the smaller set search the cache
// first (phase 1), then the larger set in global memory (phase 2).  Same two
// phases here, re-designed for B200:
//
//  * The cache is every T-th element of the larger set L (T = ceil(|L| /
//    8192)), gathered once into a compact 32 KiB array by a small kernel and
//    copied into every CTA's shared memory with 16-byte loads, so phase 2 is a
//    bounded search over a window of T elements.
//  * Each warp owns 32 J consecutive elements of the smaller set S and reads
//    them 32 at a time (coalesced); the hits of 32 elements are one ballot word,
//    written to a hit mask in global memory, and each CTA adds its hit count.
//    J (1..32) is chosen so that the grid holds about one search per thread
//    of a full B200: phase 2 is a chain of dependent global loads, so the
//    kernel is latency-bound and wants every thread in flight.
//  * Element output is a stream compaction of S by the hit mask: a scan of the
//    per-CTA counts, then every CTA writes its hits, in order, from the mask.
//    The result is ascending because S is.
// Work is |S| searches of log2(8192) shared + log2(T) global steps, so the
// technique pays off when |S| << |L| (skewed pairs); it is exact for any sizes.
#include <algorithm>

#include "si_device.cuh"
#include "si_internal.h"

namespace si {
namespace {

constexpr uint32_t kTop = 8192;             // cached samples of L (32 KiB of shared memory)
constexpr int kObsThreads = 256;
constexpr int kObsWarps = kObsThreads / 32;
constexpr size_t kObsHeader = 256;          // error words

struct ObsLayout {
    uint64_t nTop = 0, T = 0, nChunks = 0, nWords = 0;
    uint32_t J = 1;                          // mask words (of 32 elements) per warp
    uint64_t chunk = 0;                      // elements of S per CTA: kObsWarps x 32 J
    size_t off_top = 0, off_mask = 0, off_ccount = 0, off_coffset = 0, total = 0;
};

ObsLayout obs_layout(uint64_t nS, uint64_t nL, uint32_t sms) {
    ObsLayout L;
    L.T = std::max<uint64_t>(1, (nL + kTop - 1) / kTop);
    L.nTop = nL ? (nL + L.T - 1) / L.T : 0;
    const uint64_t threads = uint64_t(sms) * 2048;  // resident threads of the GPU
    while (L.J < 32 && uint64_t(L.J) * 2 * threads <= nS) L.J *= 2;
    L.chunk = uint64_t(kObsWarps) * 32 * L.J;
    L.nChunks = (nS + L.chunk - 1) / L.chunk;
    L.nWords = L.nChunks * kObsWarps * L.J;
    // offsets sized for any J, so the workspace size depends on the sizes only
    const uint64_t max_words = (nS + kObsWarps * 32 * 32 - 1) / (kObsWarps * 32 * 32) * kObsWarps * 32;
    const uint64_t max_chunks = (nS + kObsWarps * 32 - 1) / (kObsWarps * 32);
    size_t o = kObsHeader;
    L.off_top = o;
    o = align_up(o + kTop * 4, 256);
    L.off_mask = o;
    o = align_up(o + std::max(max_words, max_chunks * kObsWarps) * 4, 256);
    L.off_ccount = o;
    o = align_up(o + max_chunks * 4, 256);
    L.off_coffset = o;
    o = align_up(o + (max_chunks + 1) * 8, 256);
    L.total = o;
    return L;
}

__global__ void obs_sample_kernel(const uint32_t* __restrict__ L, uint64_t T, uint64_t nTop, uint32_t* __restrict__ top) {
    for (uint64_t w = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; w < kTop; w += uint64_t(gridDim.x) * blockDim.x)
        top[w] = w < nTop ? L[w * T] : 0xffffffffu;  // tail entries are never selected (see obs_find)
}

// Is x in L?  Phase 1: the last cached sample <= x (branch-free search over
// the kTop shared entries, of which the first nTop are real).  Phase 2: lower
// bound of x in that sample's window of L.
__device__ __forceinline__ bool obs_find(uint32_t x, const uint32_t* __restrict__ top, uint32_t nTop,
                                         const uint32_t* __restrict__ L, uint64_t nL, uint64_t T) {
    if (nTop == 0 || x < top[0]) return false;
    uint32_t pos = 0;  // invariant: top[pos] <= x
#pragma unroll
    for (uint32_t step = kTop / 2; step > 0; step >>= 1) {
        const uint32_t p = pos + step;
        pos = (p < nTop && top[p] <= x) ? p : pos;
    }
    uint64_t lo = uint64_t(pos) * T;
    uint64_t len = nL - lo < T ? nL - lo : T;  // window [lo, lo + len), L[lo] <= x
    while (len > 1) {
        const uint64_t half = len >> 1;
        const bool c = __ldg(L + lo + half) <= x;
        lo = c ? lo + half : lo;
        len = c ? len - half : half;
    }
    return __ldg(L + lo) == x;
}

// Phase 1 + 2 for one chunk of S per CTA: hit mask words, per-chunk counts;
// count-only mode adds the counts into d_count instead.
template <bool kOut>
__global__ void __launch_bounds__(kObsThreads) obs_search_kernel(const uint32_t* __restrict__ S, uint64_t nS,
                                                                 const uint32_t* __restrict__ L, uint64_t nL,
                                                                 uint64_t T, uint32_t nTop,
                                                                 const uint32_t* __restrict__ top_g,
                                                                 uint32_t* __restrict__ mask,
                                                                 uint32_t* __restrict__ ccount,
                                                                 uint64_t* __restrict__ d_count, uint64_t nChunks,
                                                                 uint32_t J) {
    __shared__ __align__(16) uint32_t top[kTop];
    __shared__ uint32_t s_warp[kObsThreads / 32];
    const uint4* src = reinterpret_cast<const uint4*>(top_g);
    uint4* dst = reinterpret_cast<uint4*>(top);
    for (uint32_t i = threadIdx.x; i < kTop / 4; i += kObsThreads) dst[i] = src[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t c = blockIdx.x; c < nChunks; c += gridDim.x) {
        const uint64_t base = (c * kObsWarps + warp) * 32 * J;
        uint32_t hits = 0;
#pragma unroll 4
        for (uint32_t j = 0; j < J; ++j) {
            const uint64_t i = base + uint64_t(j) * 32 + lane;
            const bool hit = i < nS && obs_find(__ldg(S + i), top, nTop, L, nL, T);
            const uint32_t word = __ballot_sync(kFullMask, hit);
            if (kOut && lane == 0) mask[(base >> 5) + j] = word;
            hits += lane == 0 ? __popc(word) : 0u;
        }
        if (lane == 0) s_warp[warp] = hits;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t total = 0;
            for (int w = 0; w < kObsThreads / 32; ++w) total += s_warp[w];
            if (kOut) ccount[c] = total;
            else if (total) atomicAdd(reinterpret_cast<unsigned long long*>(d_count), total);
        }
        __syncthreads();
    }
}

// Exclusive scan of the per-chunk counts (one CTA), total into d_count.
__global__ void __launch_bounds__(1024) obs_scan_kernel(const uint32_t* __restrict__ ccount, uint64_t nChunks,
                                                        uint64_t* __restrict__ coffset, uint64_t* __restrict__ d_count) {
    __shared__ uint64_t s_warp[32];
    __shared__ uint64_t s_carry;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (uint64_t b = 0; b < nChunks; b += 1024) {
        const uint64_t i = b + threadIdx.x;
        const uint64_t v = i < nChunks ? ccount[i] : 0;
        uint64_t x = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t n = __shfl_up_sync(kFullMask, x, d);
            if (lane >= d) x += n;
        }
        if (lane == 31) s_warp[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint64_t y = s_warp[lane];
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint64_t n = __shfl_up_sync(kFullMask, y, d);
                if (lane >= d) y += n;
            }
            s_warp[lane] = y;  // inclusive over warps
        }
        __syncthreads();
        const uint64_t carry = s_carry;
        const uint64_t excl = carry + (warp ? s_warp[warp - 1] : 0) + x - v;
        if (i < nChunks) coffset[i] = excl;
        __syncthreads();
        if (threadIdx.x == 0) s_carry = carry + s_warp[31];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        coffset[nChunks] = s_carry;
        *d_count = s_carry;
    }
}

// Compaction: every warp re-reads its J mask words, lane j < J takes word j
// and writes the hits of elements base + 32 j ... in order.
__global__ void __launch_bounds__(kObsThreads) obs_compact_kernel(const uint32_t* __restrict__ S,
                                                                  const uint32_t* __restrict__ mask,
                                                                  const uint32_t* __restrict__ ccount,
                                                                  const uint64_t* __restrict__ coffset,
                                                                  uint32_t* __restrict__ out, uint64_t nChunks,
                                                                  uint32_t J) {
    __shared__ uint32_t s_warp[kObsThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t c = blockIdx.x; c < nChunks; c += gridDim.x) {
        if (ccount[c] == 0) continue;  // uniform over the CTA
        const uint64_t base = (c * kObsWarps + warp) * 32 * J;
        const uint32_t word = uint32_t(lane) < J ? mask[(base >> 5) + lane] : 0u;
        const uint32_t n = __popc(word);
        const uint32_t incl = warp_inclusive_scan(n);
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        uint64_t pos = coffset[c] + incl - n;
        for (int w = 0; w < warp; ++w) pos += s_warp[w];
        uint32_t m = word;
        while (m) {
            const int x = __ffs(m) - 1;
            m &= m - 1;
            out[pos++] = __ldg(S + base + uint64_t(lane) * 32 + x);
        }
        __syncthreads();
    }
}

}  // namespace

size_t obs_workspace_size(uint64_t nA, uint64_t nB) {
    return obs_layout(std::min(nA, nB), std::max(nA, nB), 1).total;
}

si_status obs_sisi(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB, uint64_t* d_count,
                   uint32_t* d_out, void* ws, size_t ws_bytes, cudaStream_t stream) {
    // S: the smaller set (A on ties), searched for in the larger set L
    const bool a_small = nA <= nB;
    const uint32_t* S = a_small ? dA : dB;
    const uint32_t* Lp = a_small ? dB : dA;
    const uint64_t nS = a_small ? nA : nB, nL = a_small ? nB : nA;
    const ObsLayout Lo = obs_layout(nS, nL, sm_count());
    if (ws_bytes < Lo.total) return SI_ERR_WORKSPACE_TOO_SMALL;
    unsigned char* w = static_cast<unsigned char*>(ws);
    SI_CUDA_TRY(cudaMemsetAsync(w, 0, kObsHeader, stream));
    SI_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), stream));
    if (nS == 0 || nL == 0) return SI_OK;
    uint32_t* top = reinterpret_cast<uint32_t*>(w + Lo.off_top);
    uint32_t* mask = reinterpret_cast<uint32_t*>(w + Lo.off_mask);
    uint32_t* ccount = reinterpret_cast<uint32_t*>(w + Lo.off_ccount);
    uint64_t* coffset = reinterpret_cast<uint64_t*>(w + Lo.off_coffset);
    {
        PhaseTimer timer("obs_sample", stream);
        obs_sample_kernel<<<kTop / 256, 256, 0, stream>>>(Lp, Lo.T, Lo.nTop, top);
    }
    SI_LAUNCH_CHECK("obs_sample_kernel");
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(Lo.nChunks, uint64_t(sm_count()) * 8));
    {
        PhaseTimer timer("obs_search", stream);
        if (d_out)
            obs_search_kernel<true><<<grid, kObsThreads, 0, stream>>>(S, nS, Lp, nL, Lo.T, uint32_t(Lo.nTop), top,
                                                                     mask, ccount, d_count, Lo.nChunks, Lo.J);
        else
            obs_search_kernel<false><<<grid, kObsThreads, 0, stream>>>(S, nS, Lp, nL, Lo.T, uint32_t(Lo.nTop), top,
                                                                      mask, ccount, d_count, Lo.nChunks, Lo.J);
    }
    SI_LAUNCH_CHECK("obs_search_kernel");
    if (!d_out) return SI_OK;
    {
        PhaseTimer timer("obs_scan", stream);
        obs_scan_kernel<<<1, 1024, 0, stream>>>(ccount, Lo.nChunks, coffset, d_count);
    }
    SI_LAUNCH_CHECK("obs_scan_kernel");
    {
        PhaseTimer timer("obs_compact", stream);
        obs_compact_kernel<<<grid, kObsThreads, 0, stream>>>(S, mask, ccount, coffset, d_out, Lo.nChunks, Lo.J);
    }
    SI_LAUNCH_CHECK("obs_compact_kernel");
    return SI_OK;
}

}  // namespace si
