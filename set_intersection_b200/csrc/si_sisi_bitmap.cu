// si_sisi_bitmap.cu -- technique bitmap for one pair of large sorted sets
// (and SI_TECH_AUTO for pairs of similar size), plus the value-pivot split
// that the intersect-path tiles use.
//
// Replaces the single-instance path of bitmap_dynamic (src/bitmap_dynamic.cu:
// 168-176: constructBitmap over the whole universe, singleInstanceIntersect,
// thrust::reduce).  The reference sets one bit per element of A in a bitmap as
// large as the universe (2^31 bits = 256 MiB for the 2^28 x 2^28 pair) and
// probes it with every element of B from global memory.  Here the bitmaps are
// small, private to a warp and cover a window of 32768 values at a time:
//
//  bp_stream_kernel  one warp per range of the larger set X (ranges of equal
//      element count, about one per resident warp), streaming X's range and the
//      smaller set Y from the first element not below the range's start, both
//      with coalesced 16-byte loads one chunk (256 elements) ahead and bulk L2
//      prefetches four to eight chunks ahead.  Per window of values each
//      stream's elements set bits in its own 4 KiB bitmap (shared red.or, no
//      barrier: the warp owns its bitmaps); the AND of the two bitmaps is the
//      window's part of the intersection, in value order.  The next window
//      starts at the larger of the two sets' next elements, so stretches where
//      one set has no element are skipped.  Counting: popcounts.  Element
//      output: each warp writes its range's hits in order to a scratch array
//      (at the range's first Y index) and their number; the last CTA to finish
//      turns the ranges' counts into output offsets.
//  bp_copy_kernel  each range's hits from scratch to out (a warp per range),
//      and the total count.  Launched as a programmatic dependent, so its
//      launch overlaps the stream kernel's tail.
//
//  bh_stream_kernel  technique hi on the same ranges: Y in windows of 512
//      elements goes into a warp-private 2048-slot hash table (load <= 1/4),
//      the range's X elements up to the window's last value probe it; the
//      same scratch, range scan and copy kernel as the bitmap stream.
//
//  pivot_sample_kernel + pivot_split_kernel  the intersect-path tiles' split
//      (si_sisi_ip.cu): every S-th element of each set is a pivot; one warp
//      per pivot finds its rank in the merged pivot order (a merge-path search
//      over the compact samples) and its exact split in the other set (a
//      128-element probe at the interpolated position, else a warp search).
//
// X is the larger set, Y the smaller (the scratch array is as long as Y).
// Sets must be sorted and duplicate-free; this engine does not detect
// unsorted input (si_validate_sorted does).
#include <algorithm>

#include "si_device.cuh"
#include "si_internal.h"
#include "si_stream.cuh"

namespace si {
namespace {

// ------------------------------------------------------------ pivot split --
// Samples sa[k] = A[k S], sb[k] = B[k S]; clears zero[0, nzero) and the count.
__global__ void __launch_bounds__(256) pivot_sample_kernel(const uint32_t* __restrict__ A, uint64_t nA,
                                                           const uint32_t* __restrict__ B, uint64_t nB, uint64_t S,
                                                           uint32_t* __restrict__ sa, uint32_t* __restrict__ sb,
                                                           uint64_t* __restrict__ zero, uint64_t nzero,
                                                           uint64_t* __restrict__ d_count) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const uint64_t nSA = (nA + S - 1) / S, nSB = (nB + S - 1) / S;
    const uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    if (t0 == 0) *d_count = 0;
    for (uint64_t k = t0; k < nSA; k += stride) sa[k] = __ldg(A + k * S);
    for (uint64_t k = t0; k < nSB; k += stride) sb[k] = __ldg(B + k * S);
    for (uint64_t k = t0; k < nzero; k += stride) zero[k] = 0;
}

// #(O[lo, hi) < v) + lo, warp-cooperative, for a window whose elements before
// lo are < v and from hi on are >= v.  vlo = O[lo]; vhi = O[hi] when
// have_vhi.  First a 128-element probe around the position interpolated
// between vlo and vhi (one round trip for evenly spread values), else a warp
// search of the side of the probe the answer lies on.
__device__ __forceinline__ uint64_t window_rank(const uint32_t* __restrict__ O, uint64_t lo, uint64_t hi, uint32_t v,
                                                uint32_t vlo, uint32_t vhi, bool have_vhi) {
    const uint32_t lane = threadIdx.x & 31;
    constexpr uint64_t kW = 128;
    uint64_t wb = lo;
    if (hi - lo > kW) {
        uint64_t est = lo + (hi - lo) / 2;
        if (have_vhi && vhi > vlo && v >= vlo)
            est = lo + static_cast<uint64_t>(v - vlo) * (hi - lo) / (static_cast<uint64_t>(vhi) - vlo);
        wb = est > lo + kW / 2 ? est - kW / 2 : lo;
        if (wb + kW > hi) wb = hi - kW;
    }
    uint32_t c = 0, first = 0, last = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const uint64_t x = wb + 32 * r + lane;
        if (x < hi) {
            const uint32_t e = __ldg(O + x);
            c += e < v ? 1u : 0u;
            if (r == 0 && lane == 0) first = e;
            if (x == min(wb + kW, hi) - 1) last = e;
        }
    }
    c = __reduce_add_sync(kFullMask, c);
    first = __shfl_sync(kFullMask, first, 0);
    const uint32_t last_lane = static_cast<uint32_t>((min(wb + kW, hi) - 1 - wb) & 31);
    last = __shfl_sync(kFullMask, last, last_lane);
    const uint64_t wend = min(wb + kW, hi);
    if (wb > lo && first >= v)  // the answer lies before the probe
        return warp_first_true(lo, wb, [&](uint64_t x) { return __ldg(O + x) >= v; });
    if (wend < hi && last < v)  // ... or after it
        return warp_first_true(wend, hi, [&](uint64_t x) { return __ldg(O + x) >= v; });
    return wb + c;
}

// One warp per pivot rank u in [0, nSA + nSB) (thread 0 also closes the
// table): split_a[u + 1] = #A elements below the pivot's value (exact for an
// A pivot: its index), split_b[u + 1] likewise.  split[0] = (0, 0) and
// split[nP + 1] = (nA, nB).  Ties between an A and a B pivot: A first.
__global__ void __launch_bounds__(256) pivot_split_kernel(const uint32_t* __restrict__ A, uint64_t nA,
                                                          const uint32_t* __restrict__ B, uint64_t nB, uint64_t S,
                                                          const uint32_t* __restrict__ sa,
                                                          const uint32_t* __restrict__ sb,
                                                          uint64_t* __restrict__ split_a,
                                                          uint64_t* __restrict__ split_b) {
    // the dependent launch (the tile kernel) may start its set-up now; it
    // waits for this grid's completion before it reads anything written here
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");  // the samples
    const uint64_t nSA = (nA + S - 1) / S, nSB = (nB + S - 1) / S, nP = nSA + nSB;
    const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    if (tid == 0) {
        split_a[0] = 0;
        split_b[0] = 0;
        split_a[nP + 1] = nA;
        split_b[nP + 1] = nB;
    }
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t u = tid / 32; u < nP; u += nthreads / 32) {
        // i = #A pivots among the first u of the merged order: the first i in
        // [max(0, u - nSB), min(u, nSA)) whose A pivot comes after B pivot u-1-i
        const uint64_t ilo = u > nSB ? u - nSB : 0, ihi = u < nSA ? u : nSA;
        const uint64_t i = warp_first_true(ilo, ihi, [&](uint64_t x) { return sa[x] > sb[u - 1 - x]; });
        const uint64_t j = u - i;
        const uint32_t va = i < nSA ? sa[i] : 0u, vb = j < nSB ? sb[j] : 0u;
        const bool isA = i < nSA && (j >= nSB || va <= vb);
        // exact split in the other set O: #(O < v) lies in the window of O's
        // preceding pivot, [(w - 1) S, min(w S, nO))
        const uint32_t v = isA ? va : vb;
        const uint32_t* O = isA ? B : A;
        const uint32_t* SO = isA ? sb : sa;
        const uint64_t nO = isA ? nB : nA, nSO = isA ? nSB : nSA, w = isA ? j : i;
        uint64_t other = 0;
        if (w > 0) {
            const uint64_t lo = (w - 1) * S, hi = min(w * S, nO);
            other = window_rank(O, lo, hi, v, SO[w - 1], w < nSO ? SO[w] : 0u, w < nSO);
        }
        if (lane == 0) {
            split_a[u + 1] = isA ? i * S : other;
            split_b[u + 1] = isA ? other : j * S;
        }
    }
}

// ------------------------------------------------------ bitmap stream --
// values per window: 32768 (a 4 KiB bitmap per set; 16384 measured 2.4 %
// slower on the 2^28 pair: half as many chunks straddle two windows here)
constexpr uint32_t kWin = 32768;
constexpr uint32_t kWinWords = kWin / 32;
constexpr int kStWarps = 8;                     // warps per CTA
constexpr int kStBlock = kStWarps * 32;
constexpr int kStCtasPerSm = 3;                 // 24 warps per SM (85 registers each)
constexpr uint64_t kMinRange = 4096;            // X elements per warp, at least
constexpr uint32_t kBmBytes = kWinWords * 4;    // one bitmap, aligned to its size in shared memory
constexpr size_t kStSmem = size_t(kStWarps) * 2 * kBmBytes + kBmBytes;  // + the skew to a bitmap boundary

// The last CTA of a stream kernel to finish turns the ranges' counts into
// output offsets (exclusive prefix sums; 256 threads, a contiguous share of
// the ranges each).
__device__ __forceinline__ void last_cta_scan(const uint32_t* __restrict__ range_count,
                                              uint64_t* __restrict__ range_off, uint64_t nRanges,
                                              uint32_t* __restrict__ done_ctas) {
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ uint32_t s_last;
    __shared__ uint64_t s_warp[kStWarps];
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = atomicAdd(done_ctas, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const uint64_t per = (nRanges + kStBlock - 1) / kStBlock;
    const uint64_t r0 = nRanges < threadIdx.x * per ? nRanges : threadIdx.x * per;
    const uint64_t r1 = nRanges < r0 + per ? nRanges : r0 + per;
    uint64_t sum = 0;
    for (uint64_t r = r0; r < r1; ++r) sum += __ldcg(range_count + r);
    uint64_t incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint64_t n = __shfl_up_sync(kFullMask, incl, d);
        if (static_cast<int>(lane) >= d) incl += n;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint64_t before = 0;
    for (uint32_t w = 0; w < warp; ++w) before += s_warp[w];
    uint64_t off = before + incl - sum;
    for (uint64_t r = r0; r < r1; ++r) {
        range_off[r] = off;
        off += __ldcg(range_count + r);
    }
}

// One warp per range r of X: X elements [r L, (r + 1) L) and the Y elements
// from the first one not below X[r L] on.  Both streams pass through windows
// of kWin values [a, a + kWin): each window's X and Y elements set bits in the
// warp's two bitmaps, whose AND is the window's part of the intersection, in
// value order.  The next window starts at the larger of the two sets' next
// elements, so stretches where one set has no element are skipped.
// Element output: hit number k of range r goes to scratch[range_y[r] + k]
// (a range has at most as many hits as Y elements from range_y[r] on).
template <bool kOut>
__global__ void __launch_bounds__(kStBlock, kStCtasPerSm) bp_stream_kernel(
    const uint32_t* __restrict__ X, uint64_t nX, const uint32_t* __restrict__ Y, uint64_t nY, uint64_t L,
    uint64_t nRanges, uint32_t* __restrict__ range_count, uint64_t* __restrict__ range_y,
    uint64_t* __restrict__ range_off, uint32_t* __restrict__ scratch, uint64_t* __restrict__ d_count,
    uint32_t* __restrict__ done_ctas) {
    extern __shared__ __align__(16) uint32_t smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // bitmaps aligned to their size in the shared window (bit_or forms word addresses with one LOP3)
    const uint32_t skew = ((smem_addr(smem) + (kBmBytes - 1)) & ~(kBmBytes - 1)) - smem_addr(smem);
    uint32_t* bmx = smem + skew / 4 + warp * 2 * kWinWords;
    uint32_t* bmy = bmx + kWinWords;
    const uint32_t sbx = smem_addr(bmx), sby = smem_addr(bmy);
    uint4* bx4 = reinterpret_cast<uint4*>(bmx);
    uint4* by4 = reinterpret_cast<uint4*>(bmy);
    for (uint32_t i = lane; i < kWinWords / 2; i += 32) bx4[i] = make_uint4(0u, 0u, 0u, 0u);  // both bitmaps
    __syncwarp();
    const uint64_t nwarps = static_cast<uint64_t>(gridDim.x) * kStWarps;
    uint64_t my_hits = 0;
    for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * kStWarps + warp; r < nRanges; r += nwarps) {
        const uint64_t xs = r * L, xe = min(xs + L, nX);
        SetStream sx, sy;
        stream_init(sx, X, xs, xe, lane);
        const uint32_t vfirst = __ldg(X + xs);
        const uint64_t ys = warp_first_true(0, nY, [&](uint64_t i) { return __ldg(Y + i) >= vfirst; });
        uint32_t hits = 0;
        if (ys < nY) {
            stream_init(sy, Y, ys, nY, lane);
            uint32_t a = __ldg(Y + ys);  // >= vfirst: no X element below it can match
            uint32_t* dst = kOut ? scratch + ys : nullptr;
            for (;;) {
                const uint64_t e = static_cast<uint64_t>(a) + kWin;
                const uint32_t lim = e > 0xffffffffull ? static_cast<uint32_t>(0x100000000ull - a) : kWin;
                const bool more_x = stream_fill<kWinWords>(sx, sbx, a, lim, e, lane);
                const bool more_y = stream_fill<kWinWords>(sy, sby, a, lim, e, lane);
                __syncwarp();
                // AND of the window's bitmaps, a quarter (128 words) at a
                // time, lane l holding words 4 l .. 4 l + 3 of the quarter
#pragma unroll
                for (uint32_t h = 0; h < kWinWords / 128; ++h) {
                    const uint32_t i = 32 * h + lane;
                    const uint4 p = bx4[i], q = by4[i];
                    bx4[i] = make_uint4(0u, 0u, 0u, 0u);
                    by4[i] = make_uint4(0u, 0u, 0u, 0u);
                    const uint32_t m[4] = {p.x & q.x, p.y & q.y, p.z & q.z, p.w & q.w};
                    const uint32_t c = __popc(m[0]) + __popc(m[1]) + __popc(m[2]) + __popc(m[3]);
                    if constexpr (kOut) {
                        // this lane's hits go to dst[hits + (hits of the lanes before it) ...]
                        const uint32_t incl = warp_inclusive_scan(c);
                        uint32_t* o = dst + (hits + incl - c);
                        const uint32_t wbase = a + 32 * 4 * i;
#pragma unroll
                        for (uint32_t j = 0; j < 4; ++j) {
                            for (uint32_t mm = m[j]; mm; mm &= mm - 1) *o++ = wbase + 32 * j + (__ffs(mm) - 1);
                        }
                        hits += __shfl_sync(kFullMask, incl, 31);
                    } else {
                        hits += __reduce_add_sync(kFullMask, c);
                    }
                }
                __syncwarp();
                if (!more_x || !more_y) break;
                a = max(stream_first_from(sx, e), stream_first_from(sy, e));
            }
        }
        if constexpr (kOut) {
            if (lane == 0) {
                range_count[r] = hits;
                range_y[r] = ys < nY ? ys : nY;
            }
        } else {
            my_hits += hits;
        }
    }
    if constexpr (!kOut) {
        if (lane == 0 && my_hits) atomicAdd(reinterpret_cast<unsigned long long*>(d_count), my_hits);
    } else {
        last_cta_scan(range_count, range_off, nRanges, done_ctas);
    }
}

// ------------------------------------------------------------ hash stream --
// Technique hi on the same ranges (the reference's hash intersection,
// src/hi.cu:295-479, in windows): one warp per range r of X streams Y from its
// first element not below X[r L] in windows of kHashWinChunks chunks; each
// window goes into the warp's kWinHashSlots-slot table (load <= 1/4) and the
// range's X elements up to the window's last value probe it.  Element output
// as the bitmap stream's: hits in value order to scratch[range_y[r] ...].
// The value 2^32 - 1 marks empty slots; it can only be the last element of X
// and of Y, and a match of it is added at the end of the last range.
constexpr uint32_t kHashWinChunks = 2;  // 512 elements of Y per window
constexpr size_t kHashSmem = size_t(kStWarps) * kWinHashSlots * sizeof(uint32_t);
static_assert(kHashWinChunks * kChunk <= kWinHashSlots / 2, "a window fills at most half of the table");

template <bool kOut>
__global__ void __launch_bounds__(kStBlock, kStCtasPerSm) bh_stream_kernel(
    const uint32_t* __restrict__ X, uint64_t nX, const uint32_t* __restrict__ Y, uint64_t nY, uint64_t L,
    uint64_t nRanges, uint32_t* __restrict__ range_count, uint64_t* __restrict__ range_y,
    uint64_t* __restrict__ range_off, uint32_t* __restrict__ scratch, uint64_t* __restrict__ d_count,
    uint32_t* __restrict__ done_ctas) {
    extern __shared__ __align__(16) uint32_t smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t* tab = smem + warp * kWinHashSlots;
    uint4* tab4 = reinterpret_cast<uint4*>(tab);
    const bool y_top = __ldg(Y + nY - 1) == kWinHashEmpty, x_top = __ldg(X + nX - 1) == kWinHashEmpty;
    const uint64_t nYe = nY - (y_top ? 1 : 0);  // Y without 2^32 - 1
    const uint64_t nwarps = static_cast<uint64_t>(gridDim.x) * kStWarps;
    uint64_t my_hits = 0;
    for (uint64_t r = static_cast<uint64_t>(blockIdx.x) * kStWarps + warp; r < nRanges; r += nwarps) {
        const uint64_t xs = r * L, xe = min(xs + L, nX);
        const bool top_here = x_top && xe == nX;  // this range holds X's 2^32 - 1
        const uint64_t xe_e = xe - (top_here ? 1 : 0);
        uint32_t hits = 0;
        uint64_t ys = nYe;
        if (xe_e > xs && nYe > 0) {
            const uint32_t vfirst = __ldg(X + xs);
            ys = warp_first_true(0, nYe, [&](uint64_t i) { return __ldg(Y + i) >= vfirst; });
        }
        if (ys < nYe) {
            SetStream sx, sy;
            stream_init(sx, X, xs, xe_e, lane);
            stream_init(sy, Y, ys, nYe, lane);
            const uint32_t xv0 = sx.v1 - static_cast<uint32_t>(xe_e - xs);  // X's first stream position
            uint32_t* dst = kOut ? scratch + ys : nullptr;
            for (;;) {
                for (uint32_t i = lane; i < kWinHashSlots / 4; i += 32)
                    tab4[i] = make_uint4(kWinHashEmpty, kWinHashEmpty, kWinHashEmpty, kWinHashEmpty);
                __syncwarp();
                // the window: the next chunks of Y, up to its last value hi
                uint32_t hi = 0;
                bool more_y = true;
                for (uint32_t c = 0; c < kHashWinChunks && more_y; ++c) {
                    if (sy.ph == 0)
                        chunk_hash_insert(tab, sy.a0, sy.a1);
                    else
                        chunk_hash_insert(tab, sy.b0, sy.b1);
                    hi = sy.last;
                    more_y = stream_next(sy, lane);
                }
                __syncwarp();
                // the range's X elements up to hi probe it; a chunk reaching past hi stays
                bool more_x = true;
                for (;;) {
                    const uint4 g0 = sx.ph == 0 ? sx.a0 : sx.b0, g1 = sx.ph == 0 ? sx.a1 : sx.b1;
                    const uint32_t hit = chunk_hash_probe(tab, g0, g1, probe_mask(sx, g0, g1, xv0, hi, lane));
                    if constexpr (kOut) {
                        // in value order: the chunk's first half (g0, lane by lane), then its second
                        const uint32_t c0 = __popc(hit & 0xfu), c1 = __popc(hit >> 4);
                        const uint32_t i0 = warp_inclusive_scan(c0), t0 = __shfl_sync(kFullMask, i0, 31);
                        const uint32_t i1 = warp_inclusive_scan(c1), t1 = __shfl_sync(kFullMask, i1, 31);
                        uint32_t* o0 = dst + hits + i0 - c0;
                        uint32_t* o1 = dst + hits + t0 + i1 - c1;
#pragma unroll
                        for (uint32_t q = 0; q < 4; ++q)
                            if ((hit >> q) & 1u) *o0++ = comp(g0, q);
#pragma unroll
                        for (uint32_t q = 0; q < 4; ++q)
                            if ((hit >> (4 + q)) & 1u) *o1++ = comp(g1, q);
                        hits += t0 + t1;
                    } else {
                        hits += __reduce_add_sync(kFullMask, __popc(hit));
                    }
                    if (sx.last > hi) break;
                    more_x = stream_next(sx, lane);
                    if (!more_x) break;
                }
                if (!more_x || !more_y) break;
                __syncwarp();  // the probes are done before the table is cleared
            }
        }
        if (top_here && y_top) {  // 2^32 - 1 in both sets: the last hit of the last range
            if (kOut && lane == 0) scratch[ys + hits] = kWinHashEmpty;
            ++hits;
        }
        if constexpr (kOut) {
            if (lane == 0) {
                range_count[r] = hits;
                range_y[r] = ys;
            }
        } else {
            my_hits += hits;
        }
    }
    if constexpr (!kOut) {
        if (lane == 0 && my_hits) atomicAdd(reinterpret_cast<unsigned long long*>(d_count), my_hits);
    } else {
        last_cta_scan(range_count, range_off, nRanges, done_ctas);
    }
}

// -------------------------------------------------------------- copy-out --
// Range t's tile_count[t] hits at scratch[split_y[t] ...] go to
// out[tile_off[t] ...].  One warp per range, grid-stride over the ranges; the
// next range's count and offsets are loaded while the current one is copied,
// and each lane keeps 16 loads in flight.  The warp of the last range writes
// the total count.
constexpr int kCopyUnroll = 16;
__global__ void __launch_bounds__(256) bp_copy_kernel(const uint32_t* __restrict__ tile_count,
                                                      const uint64_t* __restrict__ tile_off,
                                                      const uint64_t* __restrict__ split_y, uint64_t nTiles,
                                                      const uint32_t* __restrict__ scratch, uint32_t* __restrict__ out,
                                                      uint64_t out_cap, uint64_t* __restrict__ d_count, uint32_t* err) {
    asm volatile("griddepcontrol.wait;" ::: "memory");  // the counts, offsets and hits of the tile kernel
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x / 32);
    uint64_t t = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32;
    bool overflow = false;
    uint32_t n = 0;
    uint64_t o = 0, src = 0;
    if (t < nTiles) {
        n = tile_count[t];
        o = tile_off[t];
        src = split_y[t];
    }
    while (t < nTiles) {  // warp-uniform
        const uint64_t tn = t + warps;
        uint32_t n2 = 0;
        uint64_t o2 = 0, src2 = 0;
        if (tn < nTiles) {
            n2 = tile_count[tn];
            o2 = tile_off[tn];
            src2 = split_y[tn];
        }
        if (t == nTiles - 1 && lane == 0) *d_count = o + n;
        for (uint32_t i0 = 0; i0 < n; i0 += 32 * kCopyUnroll) {
            uint32_t v[kCopyUnroll];
#pragma unroll
            for (int u = 0; u < kCopyUnroll; ++u) {
                const uint32_t i = i0 + 32 * u + lane;
                v[u] = i < n ? __ldg(scratch + src + i) : 0u;
            }
#pragma unroll
            for (int u = 0; u < kCopyUnroll; ++u) {
                const uint32_t i = i0 + 32 * u + lane;
                if (i < n) {
                    if (o + i < out_cap) out[o + i] = v[u];
                    else overflow = true;
                }
            }
        }
        t = tn;
        n = n2;
        o = o2;
        src = src2;
    }
    if (overflow) record_error(err, SI_ERR_OUTPUT_OVERFLOW, 9, 0);
}

// Workspace of the bitmap stream: header (error word, finished-CTA counter),
// per-range hit counts, Y starts and output offsets, and the scratch array of
// the hits (as long as Y).
constexpr size_t kHeaderBytes = 256;
constexpr size_t kDoneCtas = 32;  // header word: CTAs of the stream kernel that finished
constexpr uint64_t kRangesBasis = 148 * kStCtasPerSm * kStWarps;  // one range per resident warp of a B200

struct BpLayout {
    uint64_t nRanges = 0, L = 0;
    size_t off_count = 0, off_y = 0, off_off = 0, off_scratch = 0, total = 0, total_count_only = 0;
};

BpLayout make_bp_layout(uint64_t nA, uint64_t nB) {
    BpLayout L;
    const uint64_t nX = std::max(nA, nB), nY = std::min(nA, nB);
    L.L = std::max<uint64_t>(kMinRange, ((nX + kRangesBasis - 1) / kRangesBasis + 3) & ~uint64_t(3));
    L.nRanges = (nX + L.L - 1) / L.L;
    size_t o = kHeaderBytes;
    L.total_count_only = o;
    L.off_count = o;   o = align_up(o + L.nRanges * 4, 256);
    L.off_y = o;       o = align_up(o + L.nRanges * 8, 256);
    L.off_off = o;     o = align_up(o + L.nRanges * 8, 256);
    L.off_scratch = o; o = align_up(o + nY * 4, 256);
    L.total = o;
    return L;
}

}  // namespace

si_status pivot_split(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB, uint64_t S,
                      uint64_t* split_a, uint64_t* split_b, uint32_t* samples_a, uint32_t* samples_b,
                      uint64_t* zero, uint64_t nzero, uint64_t* d_count, cudaStream_t stream) {
    const uint64_t nSA = (nA + S - 1) / S, nSB = (nB + S - 1) / S, nP = nSA + nSB;
    PhaseTimer timer("sisi_split", stream);
    const uint64_t work = std::max<uint64_t>(1, std::max(std::max(nSA, nSB), nzero));
    const unsigned grid1 =
        static_cast<unsigned>(std::min<uint64_t>((work + 255) / 256, static_cast<uint64_t>(sm_count()) * 8));
    pivot_sample_kernel<<<grid1, 256, 0, stream>>>(dA, nA, dB, nB, S, samples_a, samples_b, zero, nzero, d_count);
    SI_LAUNCH_CHECK("pivot_sample_kernel");
    const unsigned grid2 = static_cast<unsigned>(
        std::min<uint64_t>((std::max<uint64_t>(1, nP) + 7) / 8, static_cast<uint64_t>(sm_count()) * 16));
    return launch_dependent(pivot_split_kernel, dim3(grid2), dim3(256), 0, stream, dA, nA, dB, nB, S,
                            static_cast<const uint32_t*>(samples_a), static_cast<const uint32_t*>(samples_b),
                            split_a, split_b);
}

size_t pivot_samples_bytes(uint64_t nA, uint64_t nB, uint64_t S) {
    return align_up(((nA + S - 1) / S) * 4, 256) + align_up(((nB + S - 1) / S) * 4, 256);
}

size_t bm_workspace_size(uint64_t nA, uint64_t nB) { return make_bp_layout(nA, nB).total; }

si_status bm_sisi(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB, uint64_t* d_count,
                  uint32_t* d_out, uint64_t out_cap, void* ws, size_t ws_bytes, cudaStream_t stream, bool hash) {
    const BpLayout L = make_bp_layout(nA, nB);
    if (ws_bytes < (d_out ? L.total : L.total_count_only)) return SI_ERR_WORKSPACE_TOO_SMALL;
    if (std::max(nA, nB) >= kMaxStream) return SI_ERR_UNSUPPORTED;
    unsigned char* w = static_cast<unsigned char*>(ws);
    // the smaller set (Y) indexes the scratch array: a range has at most as
    // many hits as Y elements from its Y start on
    const bool swap = nA < nB;
    const uint32_t* X = swap ? dB : dA;
    const uint32_t* Y = swap ? dA : dB;
    const uint64_t nX = swap ? nB : nA, nY = swap ? nA : nB;
    uint32_t* range_count = reinterpret_cast<uint32_t*>(w + L.off_count);
    uint64_t* range_y = reinterpret_cast<uint64_t*>(w + L.off_y);
    uint64_t* range_off = reinterpret_cast<uint64_t*>(w + L.off_off);
    uint32_t* scratch = reinterpret_cast<uint32_t*>(w + L.off_scratch);
    {
        PhaseTimer timer("sisi_split", stream);  // the header (error word) and the count start at zero
        SI_CUDA_TRY(cudaMemsetAsync(w, 0, kHeaderBytes, stream));
        // with element output the copy kernel writes the count; counting adds into it
        if (!d_out || nX == 0 || nY == 0) SI_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), stream));
    }
    if (nX == 0 || nY == 0) return SI_OK;
    const size_t smem = hash ? kHashSmem : kStSmem;
    auto launch = [&](auto kernel) -> si_status {
        SI_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
        const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(
            (L.nRanges + kStWarps - 1) / kStWarps, static_cast<uint64_t>(sm_count()) * kStCtasPerSm));
        PhaseTimer timer("sisi_tile", stream);
        kernel<<<grid, kStBlock, smem, stream>>>(X, nX, Y, nY, L.L, L.nRanges, range_count, range_y, range_off,
                                                 scratch, d_count, reinterpret_cast<uint32_t*>(w + kDoneCtas));
        SI_LAUNCH_CHECK(hash ? "bh_stream_kernel" : "bp_stream_kernel");
        return SI_OK;
    };
    if (!d_out) return launch(hash ? bh_stream_kernel<false> : bp_stream_kernel<false>);
    si_status st = launch(hash ? bh_stream_kernel<true> : bp_stream_kernel<true>);
    if (st != SI_OK) return st;
    PhaseTimer timer("sisi_copy", stream);
    const unsigned grid = static_cast<unsigned>(
        std::max<uint64_t>(1, std::min<uint64_t>((L.nRanges + 7) / 8, static_cast<uint64_t>(sm_count()) * 8)));
    return launch_dependent(bp_copy_kernel, dim3(grid), dim3(256), 0, stream,
                            static_cast<const uint32_t*>(range_count), static_cast<const uint64_t*>(range_off),
                            static_cast<const uint64_t*>(range_y), L.nRanges, static_cast<const uint32_t*>(scratch),
                            d_out, out_cap, d_count, reinterpret_cast<uint32_t*>(w));
}

}  // namespace si
