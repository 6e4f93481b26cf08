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
//  * Phase 2 is a chain of dependent global loads, so the kernel is
//    latency-bound and wants every thread in flight: each warp owns 32 J
//    consecutive elements of S, J (1..32) chosen so that the grid holds about
//    one search per resident thread of the search kernel (its occupancy on
//    the device).  Elements of S that fall in the same window of L share the
//    window's first probes, which then hit in cache.
//  * The hits of 32 consecutive elements are one word of a hit mask in global
//    memory; each CTA counts its chunk's hits, and the last CTA to finish
//    scans the chunk counts into output offsets.
//  * Element output is a stream compaction of S by the hit mask, a warp per
//    chunk of up to 32 mask words, lanes on bits.  The result is ascending
//    because S is.
//  * Three launches: the sample kernel (which also clears the error words and
//    the count), then the search and the compaction as programmatic
//    dependents, so each one's launch overlaps the kernel before it.
// Work is |S| searches of log2(8192) shared + log2(T) global steps, so the
// technique pays off when |S| << |L| (skewed pairs); it is exact for any sizes.
#include <algorithm>
#include <mutex>
#include <unordered_map>

#include "si_device.cuh"
#include "si_internal.h"

namespace si {
namespace {

constexpr uint32_t kTop = 8192;             // cached samples of L (32 KiB of shared memory)
constexpr int kObsThreads = 256;
constexpr int kObsWarps = kObsThreads / 32;
constexpr size_t kObsHeader = 256;          // error words
constexpr size_t kObsDone = 32;             // header word: search CTAs that finished

struct ObsLayout {
    uint64_t nTop = 0, T = 0, nChunks = 0, nWords = 0;
    uint32_t J = 1;                          // mask words per warp
    uint64_t chunk = 0;                      // elements of S per CTA: kObsThreads J
    size_t off_top = 0, off_mask = 0, off_ccount = 0, off_coffset = 0, total = 0;
};

// threads: resident threads of the search kernel on the GPU.
ObsLayout obs_layout(uint64_t nS, uint64_t nL, uint64_t threads) {
    ObsLayout L;
    L.T = std::max<uint64_t>(1, (nL + kTop - 1) / kTop);
    L.nTop = nL ? (nL + L.T - 1) / L.T : 0;
    // J elements per thread: about one search per resident thread
    while (L.J < 32 && uint64_t(L.J) * 2 * threads <= nS) L.J *= 2;
    L.chunk = uint64_t(kObsThreads) * L.J;
    L.nChunks = (nS + L.chunk - 1) / L.chunk;
    L.nWords = L.nChunks * L.chunk / 32;
    // sized for any J, so the workspace size depends on the sizes only
    const uint64_t max_words = (nS + 8191) / 8192 * 256;
    const uint64_t max_chunks = (nS + 255) / 256;
    size_t o = kObsHeader;
    L.off_top = o;
    o = align_up(o + kTop * 4, 256);
    L.off_mask = o;
    o = align_up(o + max_words * 4, 256);
    L.off_ccount = o;
    o = align_up(o + max_chunks * 4, 256);
    L.off_coffset = o;
    o = align_up(o + (max_chunks + 1) * 8, 256);
    L.total = o;
    return L;
}

// top[w] = L[w T]; also clears the workspace's error words and the count.
__global__ void obs_sample_kernel(const uint32_t* __restrict__ L, uint64_t T, uint64_t nTop, uint32_t* __restrict__ top,
                                  uint32_t* __restrict__ header, uint64_t* __restrict__ d_count) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const uint64_t t0 = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    if (t0 < kObsHeader / 4) header[t0] = 0;
    if (t0 == 0) *d_count = 0;
    for (uint64_t w = t0; w < kTop; w += uint64_t(gridDim.x) * blockDim.x)
        top[w] = w < nTop ? L[w * T] : 0xffffffffu;  // tail entries are never selected (see top_find)
}

// Phase 1: the last cached sample <= x (branch-free search over the kTop
// shared entries, of which the first nTop are real); x >= top[0].
__device__ __forceinline__ uint32_t top_find(uint32_t x, const uint32_t* __restrict__ top, uint32_t nTop) {
    uint32_t pos = 0;  // invariant: top[pos] <= x
#pragma unroll
    for (uint32_t step = kTop / 2; step > 0; step >>= 1) {
        const uint32_t p = pos + step;
        pos = (p < nTop && top[p] <= x) ? p : pos;
    }
    return pos;
}

// Is x in L?  One lane: phase 1, then the lower bound of x in its sample's
// window of L.
__device__ __forceinline__ bool obs_find(uint32_t x, const uint32_t* __restrict__ top, uint32_t nTop,
                                         const uint32_t* __restrict__ L, uint64_t nL, uint64_t T) {
    if (nTop == 0 || x < top[0]) return false;
    uint64_t lo = uint64_t(top_find(x, top, nTop)) * T;
    uint64_t len = nL - lo < T ? nL - lo : T;  // window [lo, lo + len), L[lo] <= x
    while (len > 1) {
        const uint64_t half = len >> 1;
        const bool c = __ldg(L + lo + half) <= x;
        lo = c ? lo + half : lo;
        len = c ? len - half : half;
    }
    return __ldg(L + lo) == x;
}

// Exclusive scan of the chunk counts into coffset[0, n], the total also into
// d_count; one CTA of kObsThreads threads, 8 counts per thread per round.
__device__ __forceinline__ void cta_scan_counts(const uint32_t* __restrict__ ccount, uint64_t n,
                                                uint64_t* __restrict__ coffset, uint64_t* __restrict__ d_count) {
    __shared__ uint64_t s_sum[kObsWarps];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t carry = 0;
    for (uint64_t b = 0; b < n; b += 8 * kObsThreads) {
        const uint64_t i0 = b + 8 * uint64_t(threadIdx.x);
        uint32_t v[8];
        uint64_t sum = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            v[q] = i0 + q < n ? __ldcg(ccount + i0 + q) : 0u;
            sum += v[q];
        }
        uint64_t incl = sum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint64_t t = __shfl_up_sync(kFullMask, incl, d);
            if (static_cast<int>(lane) >= d) incl += t;
        }
        if (lane == 31) s_sum[warp] = incl;
        __syncthreads();
        uint64_t off = carry + incl - sum, total = 0;
#pragma unroll
        for (int w = 0; w < kObsWarps; ++w) {
            off += w < static_cast<int>(warp) ? s_sum[w] : 0ull;
            total += s_sum[w];
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            if (i0 + q < n) coffset[i0 + q] = off;
            off += v[q];
        }
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        coffset[n] = carry;
        *d_count = carry;
    }
}

// Phase 1 + 2 for one chunk of S per CTA: hit mask words and chunk counts,
// which the last CTA to finish scans into offsets; count-only mode adds the
// counts into d_count instead.
constexpr int kObsSearchCtasPerSm = 6;  // 40 registers: 6 CTAs of 256 threads and 32 KiB per SM
template <bool kOut>
__global__ void __launch_bounds__(kObsThreads, kObsSearchCtasPerSm) obs_search_kernel(const uint32_t* __restrict__ S, uint64_t nS,
                                                                 const uint32_t* __restrict__ L, uint64_t nL,
                                                                 uint64_t T, uint32_t nTop,
                                                                 const uint32_t* __restrict__ top_g,
                                                                 uint32_t* __restrict__ mask,
                                                                 uint32_t* __restrict__ ccount,
                                                                 uint64_t* __restrict__ coffset,
                                                                 uint64_t* __restrict__ d_count, uint64_t nChunks,
                                                                 uint32_t J, uint32_t* __restrict__ done) {
    __shared__ __align__(16) uint32_t top[kTop];
    __shared__ uint32_t s_warp[kObsWarps];
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");  // the samples, the cleared count and error words
    {
        // all of a thread's 16-byte loads in flight before its stores
        constexpr int kPer = kTop / 4 / kObsThreads;
        const uint4* src = reinterpret_cast<const uint4*>(top_g);
        uint4* dst = reinterpret_cast<uint4*>(top);
        uint4 t[kPer];
#pragma unroll
        for (int q = 0; q < kPer; ++q) t[q] = __ldcg(src + threadIdx.x + q * kObsThreads);
#pragma unroll
        for (int q = 0; q < kPer; ++q) dst[threadIdx.x + q * kObsThreads] = t[q];
    }
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t c = blockIdx.x; c < nChunks; c += gridDim.x) {
        const uint64_t base = (c * kObsWarps + warp) * 32 * J;
        uint32_t hits = 0;
#pragma unroll 1
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
            for (int w = 0; w < kObsWarps; ++w) total += s_warp[w];
            if (kOut) ccount[c] = total;
            else if (total) atomicAdd(reinterpret_cast<unsigned long long*>(d_count), total);
        }
        __syncthreads();
    }
    if constexpr (kOut) {
        __shared__ uint32_t s_last;
        if (threadIdx.x == 0) {
            __threadfence();
            s_last = atomicAdd(done, 1u) == gridDim.x - 1;
        }
        __syncthreads();
        if (!s_last) return;
        __threadfence();
        cta_scan_counts(ccount, nChunks, coffset, d_count);
    }
}

// Compaction.  Chunk c's W mask words start at its offset coffset[c].  With
// W <= 32 a warp takes a chunk (lane j word j); with W = 64..256 W / 32 warps
// of a CTA take one, 32 words each, and add the hits of the warps before
// them.  The warp then writes its words' hits word by word: lane b copies
// element 32 w + b when bit b of word w is set, so loads of S and stores of
// out are coalesced.
__global__ void __launch_bounds__(kObsThreads) obs_compact_kernel(const uint32_t* __restrict__ S,
                                                                  const uint32_t* __restrict__ mask,
                                                                  const uint64_t* __restrict__ coffset,
                                                                  uint32_t* __restrict__ out, uint64_t nChunks,
                                                                  uint32_t W) {
    asm volatile("griddepcontrol.wait;" ::: "memory");  // the mask and the offsets
    __shared__ uint32_t s_warp[kObsWarps];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t seg = W < 32 ? W : 32;                       // words per warp
    const uint32_t warps_per_chunk = W <= 32 ? 1 : W / 32;
    const uint32_t chunks_per_cta = kObsWarps / warps_per_chunk;
    const uint32_t part = warp % warps_per_chunk;
    const uint64_t nUnits = (nChunks + chunks_per_cta - 1) / chunks_per_cta;
    for (uint64_t u = blockIdx.x; u < nUnits; u += gridDim.x) {
        const uint64_t c = u * chunks_per_cta + warp / warps_per_chunk;
        const bool have = c < nChunks;  // warp-uniform
        const uint64_t w0 = c * W + part * 32;
        const uint32_t word = have && lane < seg ? __ldg(mask + w0 + lane) : 0u;
        const uint32_t n = __popc(word);
        const uint32_t incl = warp_inclusive_scan(n);
        uint64_t base = 0;
        if (warps_per_chunk > 1) {
            if (lane == 31) s_warp[warp] = incl;
            __syncthreads();
            for (uint32_t q = warp - part; q < warp; ++q) base += s_warp[q];
        }
        if (have) {
            const uint64_t mine = __ldg(coffset + c) + base + incl - n;  // offset of word `lane`
            const uint32_t below = (1u << lane) - 1u;
            for (uint32_t i = 0; i < seg; ++i) {
                const uint32_t wd = __shfl_sync(kFullMask, word, i);
                if (wd == 0) continue;  // warp-uniform
                const uint64_t o = __shfl_sync(kFullMask, mine, i);
                if ((wd >> lane) & 1u) out[o + __popc(wd & below)] = __ldg(S + (w0 + i) * 32 + lane);
            }
        }
        if (warps_per_chunk > 1) __syncthreads();
    }
}

// Resident threads of the search kernel (with or without element output) on
// the current device, cached per device.
uint64_t obs_resident_threads(bool out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
    static std::mutex mu;
    static std::unordered_map<int, uint64_t> cache[2];
    std::lock_guard<std::mutex> lk(mu);
    const auto it = cache[out].find(dev);
    if (it != cache[out].end()) return it->second;
    int per_sm = 0;
    const cudaError_t e = out ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, obs_search_kernel<true>,
                                                                              kObsThreads, 0)
                              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, obs_search_kernel<false>,
                                                                              kObsThreads, 0);
    if (e != cudaSuccess || per_sm <= 0) {
        (void)cudaGetLastError();
        per_sm = 1;
    }
    const uint64_t r = uint64_t(per_sm) * kObsThreads * uint64_t(sm_count());
    cache[out][dev] = r;
    return r;
}

}  // namespace

size_t obs_workspace_size(uint64_t nA, uint64_t nB) {
    return obs_layout(std::min(nA, nB), std::max(nA, nB), 1).total;  // the sizes do not depend on the threads
}

si_status obs_sisi(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB, uint64_t* d_count,
                   uint32_t* d_out, void* ws, size_t ws_bytes, cudaStream_t stream) {
    // S: the smaller set (A on ties), searched for in the larger set L
    const bool a_small = nA <= nB;
    const uint32_t* S = a_small ? dA : dB;
    const uint32_t* Lp = a_small ? dB : dA;
    const uint64_t nS = a_small ? nA : nB, nL = a_small ? nB : nA;
    const ObsLayout Lo = obs_layout(nS, nL, obs_resident_threads(d_out != nullptr));
    if (ws_bytes < Lo.total) return SI_ERR_WORKSPACE_TOO_SMALL;
    unsigned char* w = static_cast<unsigned char*>(ws);
    if (nS == 0 || nL == 0) {
        SI_CUDA_TRY(cudaMemsetAsync(w, 0, kObsHeader, stream));
        SI_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), stream));
        return SI_OK;
    }
    uint32_t* top = reinterpret_cast<uint32_t*>(w + Lo.off_top);
    uint32_t* mask = reinterpret_cast<uint32_t*>(w + Lo.off_mask);
    uint32_t* ccount = reinterpret_cast<uint32_t*>(w + Lo.off_ccount);
    uint64_t* coffset = reinterpret_cast<uint64_t*>(w + Lo.off_coffset);
    uint32_t* done = reinterpret_cast<uint32_t*>(w + kObsDone);
    {
        PhaseTimer timer("obs_sample", stream);
        obs_sample_kernel<<<kTop / 256, 256, 0, stream>>>(Lp, Lo.T, Lo.nTop, top, reinterpret_cast<uint32_t*>(w),
                                                           d_count);
    }
    SI_LAUNCH_CHECK("obs_sample_kernel");
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(Lo.nChunks, uint64_t(sm_count()) * 8));
    {
        PhaseTimer timer("obs_search", stream);
        const si_status st =
            d_out ? launch_dependent(obs_search_kernel<true>, dim3(grid), dim3(kObsThreads), 0, stream, S, nS, Lp, nL,
                                     Lo.T, uint32_t(Lo.nTop), static_cast<const uint32_t*>(top), mask, ccount,
                                     coffset, d_count, Lo.nChunks, Lo.J, done)
                  : launch_dependent(obs_search_kernel<false>, dim3(grid), dim3(kObsThreads), 0, stream, S, nS, Lp,
                                     nL, Lo.T, uint32_t(Lo.nTop), static_cast<const uint32_t*>(top), mask, ccount,
                                     coffset, d_count, Lo.nChunks, Lo.J, done);
        if (st != SI_OK) return st;
    }
    if (!d_out) return SI_OK;
    const uint32_t W = static_cast<uint32_t>(Lo.chunk / 32);  // mask words per chunk
    const uint64_t units = (Lo.nChunks + (W <= 32 ? kObsWarps : kObsWarps / (W / 32)) - 1) /
                           (W <= 32 ? kObsWarps : kObsWarps / (W / 32));
    PhaseTimer timer("obs_compact", stream);
    return launch_dependent(obs_compact_kernel,
                            dim3(static_cast<unsigned>(std::min<uint64_t>(units, uint64_t(sm_count()) * 8))),
                            dim3(kObsThreads), 0, stream, S, static_cast<const uint32_t*>(mask),
                            static_cast<const uint64_t*>(coffset), d_out, Lo.nChunks, W);
}

}  // namespace si
