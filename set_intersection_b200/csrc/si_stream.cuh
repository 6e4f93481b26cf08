// si_stream.cuh -- a sorted set read by one warp as a stream of 256-element
// chunks, and the window bitmaps and window hash tables built from such
// streams: the building blocks of the single-pair bitmap and hash engines
// (si_sisi_bitmap.cu) and of the batched pairs' window techniques
// (si_batch.cu).
#pragma once

#include <cstdint>

#include "si_device.cuh"

namespace si {

constexpr uint32_t kChunk = 256;                      // elements per chunk: two 16-byte groups per lane
constexpr uint64_t kMaxStream = (1ull << 32) - 1024;  // stream positions (and 2 chunks ahead) are 32-bit

// First index i in [lo, hi) with pred(i) true, or hi; pred is monotone
// (false ... false true ... true).  Warp-cooperative: every lane passes the
// same lo, hi and gets the same result.  Each round probes 32 evenly spaced
// positions (one per lane) and keeps the gap between the last false and the
// first true probe.  pred is only evaluated at indices in [lo, hi), and the
// result stays in [lo, hi] even when pred is not monotone (unsorted input).
template <class Pred>
__device__ __forceinline__ uint64_t warp_first_true(uint64_t lo, uint64_t hi, Pred pred) {
    const uint32_t lane = threadIdx.x & 31;
    while (hi - lo > 32) {
        const uint64_t step = (hi - lo + 31) / 32;
        const uint64_t q = lo + lane * step;
        const bool valid = q < hi;
        const uint32_t vm = __ballot_sync(kFullMask, valid);
        const uint32_t fm = __ballot_sync(kFullMask, valid && !pred(q));
        const uint32_t c = __popc(fm), nv = __popc(vm);
        if (c == 0) return lo;
        const uint64_t new_hi = c < nv ? lo + c * step : hi;
        lo = lo + (c - 1) * step + 1;
        hi = new_hi;
    }
    const uint64_t q = lo + lane;
    const uint32_t fm = __ballot_sync(kFullMask, q < hi && !pred(q));
    return lo + __popc(fm);
}

// One sorted set read by a warp as chunks of 256 elements: lane l holds the
// 16-byte groups at positions pc + 4 l and pc + 128 + 4 l of a 16-byte aligned
// base.  Two register buffers alternate (ph = 0: the current chunk is in a,
// the next one in b), so moving on copies nothing; the chunks four to eight
// ahead are prefetched into L2 every fourth chunk.  The elements of the stream
// are positions [v0, v1) (v0 < 4).  Positions before v0 in the first chunk hold
// a copy of the first element, and positions from v1 on in the last chunk a
// copy of the last, so every position of a chunk is an element of the set
// (setting a bit twice is harmless) and nothing checks positions.  Loads past
// the last group read the last group again (always a valid address).
// Positions are 32-bit: a stream is shorter than 2^32 - 1024.
struct SetStream {
    const uint32_t* base;
    uint32_t v1, pc, ph;
    uint4 a0, a1, b0, b1;
    uint32_t last;  // the current chunk's last element (its largest, in a sorted set)
};

__device__ __forceinline__ uint4 ld_group(const SetStream& s, uint32_t p) {
    const uint32_t pend = (s.v1 - 1) & ~3u;  // the last group that holds elements
    return __ldcs(reinterpret_cast<const uint4*>(s.base + min(p, pend)));
}

__device__ __forceinline__ uint32_t comp(const uint4& v, uint32_t q) {
    return q == 0 ? v.x : q == 1 ? v.y : q == 2 ? v.z : v.w;
}

__device__ __forceinline__ void set_comp(uint4& v, uint32_t q, uint32_t x) {
    v.x = q == 0 ? x : v.x;
    v.y = q == 1 ? x : v.y;
    v.z = q == 2 ? x : v.z;
    v.w = q == 3 ? x : v.w;
}

// Lane 0 asks the bulk-copy engine to bring chunks [p, p + 4) (the part that
// holds elements) into L2; one predicated instruction, no branch.
__device__ __forceinline__ void prefetch_l2(const SetStream& s, uint32_t p, uint32_t lead) {
    const uint32_t bytes = (min(p + 4 * kChunk, (s.v1 + 3) & ~3u) - p) * 4;
    asm volatile("{\n\t.reg .pred l, q;\n\t"
                 "setp.ne.u32 l, %3, 0;\n\t"
                 "setp.lt.and.u32 q, %0, %1, l;\n\t"
                 "@q cp.async.bulk.prefetch.L2.global [%2], %4;\n\t}" ::"r"(p),
                 "r"(s.v1), "l"(s.base + p), "r"(lead), "r"(bytes)
                 : "memory");
}

// The last element of the chunk at pc held in (g0, g1); in the stream's last
// chunk the positions from v1 on get copies of it.
__device__ __forceinline__ uint32_t chunk_settle(uint4& g0, uint4& g1, uint32_t pc, uint32_t v1, uint32_t lane) {
    if (pc + kChunk <= v1) return __shfl_sync(kFullMask, g1.w, 31);
    const uint32_t lp = v1 - 1 - pc;  // < 256
    const uint32_t last = __shfl_sync(kFullMask, comp(lp >= 128 ? g1 : g0, lp & 3), (lp & 127) >> 2);
#pragma unroll
    for (uint32_t q = 0; q < 4; ++q) {
        if (pc + 4 * lane + q >= v1) set_comp(g0, q, last);
        if (pc + 128 + 4 * lane + q >= v1) set_comp(g1, q, last);
    }
    return last;
}

__device__ __forceinline__ void stream_init(SetStream& s, const uint32_t* set, uint64_t i0, uint64_t i1,
                                            uint32_t lane) {
    const uint64_t p0 = i0 + ((reinterpret_cast<uintptr_t>(set) & 15u) >> 2);  // from the aligned base below set
    s.base = set - (p0 - i0) + (p0 & ~uint64_t(3));
    const uint32_t v0 = static_cast<uint32_t>(p0 & 3);
    s.v1 = static_cast<uint32_t>(v0 + (i1 - i0));
    s.pc = 0;
    s.ph = 0;
    s.a0 = ld_group(s, 4 * lane);
    s.a1 = ld_group(s, 128 + 4 * lane);
    s.b0 = ld_group(s, kChunk + 4 * lane);
    s.b1 = ld_group(s, kChunk + 128 + 4 * lane);
    prefetch_l2(s, 2 * kChunk, lane == 0);
    // the first chunk: positions before v0 get copies of the first element
    const uint32_t first = __shfl_sync(kFullMask, comp(s.a0, v0), 0);
    if (lane == 0) {
#pragma unroll
        for (uint32_t q = 0; q < 3; ++q)
            if (q < v0) set_comp(s.a0, q, first);
    }
    s.last = chunk_settle(s.a0, s.a1, 0, s.v1, lane);
}

// Moves to the next chunk (false: there is none); the buffer it leaves takes
// the chunk after that.  kFromA: the current chunk is in a (ph == 0).
template <bool kFromA>
__device__ __forceinline__ bool stream_advance(SetStream& s, uint32_t lane) {
    if (s.pc + kChunk >= s.v1) return false;
    s.pc += kChunk;
    const uint32_t p = s.pc + kChunk + 4 * lane;
    if constexpr (kFromA) {
        s.a0 = ld_group(s, p);
        s.a1 = ld_group(s, p + 128);
        s.last = chunk_settle(s.b0, s.b1, s.pc, s.v1, lane);
        s.ph = 1;
    } else {
        s.b0 = ld_group(s, p);
        s.b1 = ld_group(s, p + 128);
        s.last = chunk_settle(s.a0, s.a1, s.pc, s.v1, lane);
        s.ph = 0;
    }
    if (((s.pc / kChunk) & 3) == 2) prefetch_l2(s, s.pc + 4 * kChunk, lane == 0);
    return true;
}

// Sets bit o (< 32 kWords) of the kWords-word bitmap at shared-window address
// bm, which is aligned to its size: the word's address is one LOP3 of bm and
// o >> 3.
template <uint32_t kWords>
__device__ __forceinline__ void bit_or(uint32_t bm, uint32_t o) {
    static_assert((kWords & (kWords - 1)) == 0, "the bitmap is a power of two of words");
    // ordered before the AND pass's loads by the __syncwarp between them
    asm volatile("red.shared.or.b32 [%0], %1;" ::"r"(bm | ((o >> 3) & (4 * kWords - 4))),
                 "r"(__funnelshift_l(0u, 1u, o)));
}

// Sets the bits of the chunk's elements v with a <= v < a + lim (lim = the
// window, 32 kWords values, or 2^32 - a for the top window, so that no smaller
// value wraps into it).  bm: shared-window address of the bitmap.
template <uint32_t kWords>
__device__ __forceinline__ void chunk_insert(const uint4& g0, const uint4& g1, uint32_t last, uint32_t bm,
                                             uint32_t a, uint32_t lim) {
    if (__all_sync(kFullMask, g0.x >= a && last - a < lim)) {  // the whole chunk lies in the window
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) bit_or<kWords>(bm, comp(g0, q) - a);
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) bit_or<kWords>(bm, comp(g1, q) - a);
    } else {
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) {
            const uint32_t o0 = comp(g0, q) - a, o1 = comp(g1, q) - a;
            if (o0 < lim) bit_or<kWords>(bm, o0);
            if (o1 < lim) bit_or<kWords>(bm, o1);
        }
    }
}

// Inserts the stream's chunks into the bitmap until one reaches past e (it
// stays current: its later elements belong to later windows); false when the
// stream ran out.
template <uint32_t kWords>
__device__ __forceinline__ bool stream_fill(SetStream& s, uint32_t bm, uint32_t a, uint32_t lim, uint64_t e,
                                            uint32_t lane) {
    for (;;) {  // the buffers alternate: a, b, a, ...
        if (s.ph == 0) {
            chunk_insert<kWords>(s.a0, s.a1, s.last, bm, a, lim);
            if (__all_sync(kFullMask, s.last >= e)) return true;
            if (!stream_advance<true>(s, lane)) return false;
        }
        chunk_insert<kWords>(s.b0, s.b1, s.last, bm, a, lim);
        if (__all_sync(kFullMask, s.last >= e)) return true;
        if (!stream_advance<false>(s, lane)) return false;
    }
}

// The smallest element of the current chunk that is >= e (the chunk's last
// element is >= e).
__device__ __forceinline__ uint32_t chunk_first_from(const uint4& g0, const uint4& g1, uint64_t e) {
    uint32_t m = 0xffffffffu;
#pragma unroll
    for (uint32_t q = 0; q < 4; ++q) {
        const uint32_t v0 = comp(g0, q), v1 = comp(g1, q);
        m = v0 >= e ? min(m, v0) : m;
        m = v1 >= e ? min(m, v1) : m;
    }
    return __reduce_min_sync(kFullMask, m);
}

__device__ __forceinline__ uint32_t stream_first_from(const SetStream& s, uint64_t e) {
    return s.ph == 0 ? chunk_first_from(s.a0, s.a1, e) : chunk_first_from(s.b0, s.b1, e);
}

// ------------------------------------------------------------ window hash --
// A warp-private open-addressing table of a window of one stream's elements,
// probed by the other stream's chunks.
constexpr uint32_t kWinHashSlots = 2048;          // per warp: 8 KiB
constexpr uint32_t kWinHashEmpty = 0xffffffffu;   // the empty slot (that value is matched apart)

__device__ __forceinline__ uint32_t win_hash_slot(uint32_t v) {  // Fibonacci hashing to 11 bits
    return (v * 2654435761u) >> 21;
}

// Inserts the chunk's elements (8 per lane; repeated values are kept once).
// A window holds at most kWinHashSlots / 2 distinct values, so every probe
// sequence meets an empty slot.
__device__ __forceinline__ void chunk_hash_insert(uint32_t* tab, const uint4& g0, const uint4& g1) {
    uint32_t v[8] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w}, h[8];
    bool left[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        h[q] = win_hash_slot(v[q]);
        const uint32_t old = atomicCAS(tab + h[q], kWinHashEmpty, v[q]);
        left[q] = old != kWinHashEmpty && old != v[q];
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        while (left[q]) {
            h[q] = (h[q] + 1) & (kWinHashSlots - 1);
            const uint32_t old = atomicCAS(tab + h[q], kWinHashEmpty, v[q]);
            left[q] = old != kWinHashEmpty && old != v[q];
        }
    }
}

// Matches among the chunk's elements whose bit is set in `valid` (bit q: g0's
// component q, bit 4 + q: g1's), as a mask in the same bit order.  No element
// is kWinHashEmpty.
__device__ __forceinline__ uint32_t chunk_hash_probe(const uint32_t* tab, const uint4& g0, const uint4& g1,
                                                     uint32_t valid) {
    const uint32_t v[8] = {g0.x, g0.y, g0.z, g0.w, g1.x, g1.y, g1.z, g1.w};
    uint32_t h[8], hit = 0;
    bool left[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        h[q] = win_hash_slot(v[q]);
        const uint32_t t = tab[h[q]];
        const bool on = (valid >> q) & 1u;
        hit |= (on && t == v[q] ? 1u : 0u) << q;
        left[q] = on && t != v[q] && t != kWinHashEmpty;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        while (left[q]) {
            h[q] = (h[q] + 1) & (kWinHashSlots - 1);
            const uint32_t t = tab[h[q]];
            hit |= (t == v[q] ? 1u : 0u) << q;
            left[q] = t != v[q] && t != kWinHashEmpty;
        }
    }
    return hit;
}

// Which of the chunk at s.pc this lane probes: stream positions in
// [v0, s.v1) (the head and tail copies are not elements of their own) whose
// value is <= hi (the later ones belong to the next window).
__device__ __forceinline__ uint32_t probe_mask(const SetStream& s, const uint4& g0, const uint4& g1, uint32_t v0,
                                               uint32_t hi, uint32_t lane) {
    if ((s.pc != 0 || v0 == 0) && s.pc + kChunk <= s.v1 && s.last <= hi) return 0xffu;
    uint32_t m = 0;
#pragma unroll
    for (uint32_t q = 0; q < 4; ++q) {
        const uint32_t p0 = s.pc + 4 * lane + q, p1 = p0 + 128;
        m |= (p0 >= v0 && p0 < s.v1 && comp(g0, q) <= hi ? 1u : 0u) << q;
        m |= (p1 >= v0 && p1 < s.v1 && comp(g1, q) <= hi ? 1u : 0u) << (4 + q);
    }
    return m;
}

__device__ __forceinline__ bool stream_next(SetStream& s, uint32_t lane) {
    return s.ph == 0 ? stream_advance<true>(s, lane) : stream_advance<false>(s, lane);
}

}  // namespace si
