// si_sisi_bitmap.cu -- technique bitmap for one pair of large sorted sets
// (and SI_TECH_AUTO for pairs of similar size), plus the value-pivot split
// shared with the intersect-path tiles.
//
// Replaces the single-instance path of bitmap_dynamic (src/bitmap_dynamic.cu:
// 168-176: constructBitmap over the whole universe, singleInstanceIntersect,
// thrust::reduce).  The reference sets one bit per element of A in a bitmap as
// large as the universe (2^31 bits = 256 MiB for the 2^28 x 2^28 pair) and
// probes it with every element of B from global memory.  Here the bitmaps are
// small and private to a warp, and live in shared memory:
//
//  K1  pivot_split_kernel: every S-th element of each set is a pivot; one warp
//      per pivot finds its rank in the merged pivot order (a merge-path search
//      over the two sample sequences) and its exact split in the other set (a
//      search inside an S-element window).  Consecutive pivots bound a tile to
//      <= S elements of each set; a tile boundary is a value, so an equal pair
//      is never split.  Also clears the workspace header and the count.
//  K2  bp_tile_kernel, persistent, one CTA of 32 warps per SM:
//        warp 30 lane 0  stages tiles (ticket order) into a 160 KiB shared ring
//                        with bulk copies (TMA), several tiles ahead;
//        warp 31         per staged tile, the Y start of every consumer's range
//                        (a binary search per lane in the staged Y part);
//        warps 0..29     consumer w takes the X elements [w nx/30, (w+1) nx/30)
//                        of the tile, sets their bits in its own 2 KiB bitmap
//                        (values v0 .. v0 + 16383, v0 its first element), probes
//                        it with the Y elements of its value range and writes
//                        the hits in order (one ballot per 32 probes).
//      No barrier between consumers: each one only waits for its tile's
//      boundaries and releases the ring slot when done.  The hits of warp w of
//      tile t -- a "unit" -- go to scratch[first Y index of the unit + rank]
//      and their number to unit_count[t * 30 + w].
//  K3  exclusive scan of the unit counts (CUB).
//  K4  bp_copy_kernel: the units' hits from scratch to out, 32 units per warp
//      as one contiguous output run (coalesced stores), and the total count.
// Count-only mode runs K1 and K2 and adds the hits into d_count.
//
// X is the larger set (its tile part is split by index and built), Y the
// smaller (probed; the scratch array is as long as Y).  A consumer whose X
// elements span 16384 values or more searches each Y element in its X run
// instead (binary search in shared memory).
#include <algorithm>
#include <cub/device/device_scan.cuh>

#include "si_device.cuh"
#include "si_internal.h"

namespace si {
namespace {

// ----------------------------------------------------------------- K1 --
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

// One warp per pivot rank u in [0, nSA + nSB) (thread 0 also closes the
// table): split_a[u + 1] = #A elements below the pivot's value (exact for an
// A pivot: its index), split_b[u + 1] likewise.  split[0] = (0, 0) and
// split[nP + 1] = (nA, nB).  Ties between an A and a B pivot: A first.
__global__ void __launch_bounds__(256) pivot_split_kernel(const uint32_t* __restrict__ A, uint64_t nA,
                                                          const uint32_t* __restrict__ B, uint64_t nB, uint64_t S,
                                                          uint64_t* __restrict__ split_a, uint64_t* __restrict__ split_b,
                                                          uint64_t* __restrict__ zero, uint64_t nzero,
                                                          uint64_t* __restrict__ d_count) {
    // the dependent launch (the tile kernel) may start its set-up now; it
    // waits for this grid's completion before it reads anything written here
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const uint64_t nSA = (nA + S - 1) / S, nSB = (nB + S - 1) / S, nP = nSA + nSB;
    const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t nthreads = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t k = tid; k < nzero; k += nthreads) zero[k] = 0;
    if (tid == 0) {
        *d_count = 0;
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
        const uint64_t i = warp_first_true(ilo, ihi, [&](uint64_t x) {
            return __ldg(A + x * S) > __ldg(B + (u - 1 - x) * S);
        });
        const uint64_t j = u - i;
        uint32_t va = 0, vb = 0;
        if (lane == 0 && i < nSA) va = __ldg(A + i * S);
        if (lane == 1 && j < nSB) vb = __ldg(B + j * S);
        va = __shfl_sync(kFullMask, va, 0);
        vb = __shfl_sync(kFullMask, vb, 1);
        const bool isA = i < nSA && (j >= nSB || va <= vb);
        // exact split in the other set: #(elements < v) lies in the window of
        // the other set's preceding pivot, [(w - 1) S, min(w S, n))
        const uint32_t v = isA ? va : vb;
        const uint32_t* O = isA ? B : A;
        const uint64_t nO = isA ? nB : nA, w = isA ? j : i;
        uint64_t other = 0;
        if (w > 0) {
            const uint64_t lo = (w - 1) * S, hi = min(w * S, nO);
            other = warp_first_true(lo, hi, [&](uint64_t x) { return __ldg(O + x) >= v; });
        }
        if (lane == 0) {
            split_a[u + 1] = isA ? i * S : other;
            split_b[u + 1] = isA ? other : j * S;
        }
    }
}

// ----------------------------------------------------------------- K2 --
constexpr uint64_t kBpS = 16384;              // pivot stride: a tile holds <= 16384 elements per set
constexpr int kBpWarps = 30;                  // consumer warps
constexpr int kBpStageWarp = 30;              // lane 0 stages
constexpr int kBpBoundWarp = 31;              // per-tile consumer boundaries
constexpr int kBpBlock = 32 * 32;
constexpr uint32_t kBpWords = 512;            // per-consumer bitmap: 16384 values, 2 KiB
constexpr uint32_t kBpSpan = kBpWords * 32;
constexpr uint32_t kBpRing = 40960;           // u32: 160 KiB, about 2.5 average tiles
constexpr int kBpSlots = 8;
constexpr size_t kBpSmem = (size_t(kBpRing) + size_t(kBpWarps) * kBpWords) * sizeof(uint32_t);
constexpr uint32_t kEndTile = 0xffffffffu;
static_assert(2 * (kBpS + 4) <= kBpRing, "one tile's aligned supersets must fit the ring");
static_assert(kBpWarps + 1 <= 32, "one boundary per lane of the boundary warp");

struct BpDesc {
    uint64_t y0;          // global index of the tile's first Y element
    uint32_t tile;
    uint32_t offX, offY;  // ring index of element 0 of the staged X / Y part
    uint32_t misX;        // X element 0's position in its 16-byte block
    uint32_t nx, ny;
};

// Sets the bits of X elements [i0, i1) (values v0 .. v0 + span, span <
// kBpSpan), read as the 16-byte groups of the staged part that hold them.
// A group's words outside [i0, i1) are skipped by their index (at the ends of
// the arrays those words are not elements at all).
__device__ __forceinline__ void bp_build(uint32_t* bm, const uint32_t* ring, const BpDesc& d, uint32_t i0,
                                         uint32_t i1, uint32_t v0, uint32_t lane) {
    const uint4* g4 = reinterpret_cast<const uint4*>(ring + (d.offX - d.misX));
    const uint32_t e_first = d.misX + i0, n = i1 - i0;
    const uint32_t g_lo = e_first >> 2, g_hi = (d.misX + i1 - 1) >> 2;
#pragma unroll 2
    for (uint32_t g = g_lo + lane; g <= g_hi; g += 32) {
        const uint4 v = g4[g];
        const uint32_t e = 4 * g - e_first;  // wraps for the first group's leading words: then >= n
        const uint32_t vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (e + q < n) {
                const uint32_t o = vv[q] - v0;
                atomicOr(bm + (o >> 5), 1u << (o & 31));
            }
        }
    }
}

// Probes Y elements [j0, j1) (all >= v0) against the bitmap; hit number r goes
// to dst[r] (when kOut).  Returns the number of hits.
template <bool kOut>
__device__ __forceinline__ uint32_t bp_probe(const uint32_t* bm, const uint32_t* sy, uint32_t j0, uint32_t j1,
                                             uint32_t v0, uint32_t span, uint32_t* dst, uint32_t lane) {
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t pos = 0;
#pragma unroll 2
    for (uint32_t j = j0; j < j1; j += 32) {
        const uint32_t jj = j + lane;
        bool hit = false;
        uint32_t b = 0;
        if (jj < j1) {
            b = sy[jj];
            const uint32_t o = b - v0;
            if (o <= span) hit = (bm[o >> 5] >> (o & 31)) & 1u;
        }
        const uint32_t m = __ballot_sync(kFullMask, hit);
        if (kOut && hit) dst[pos + __popc(m & lt)] = b;
        pos += __popc(m);
    }
    return pos;
}

// Consumers whose X run spans too many values for the bitmap: every Y element
// of [j0, j1) is searched in X elements [i0, i1) (binary search in shared memory).
template <bool kOut>
__device__ uint32_t bp_search(const uint32_t* sx, uint32_t i0, uint32_t i1, const uint32_t* sy, uint32_t j0,
                              uint32_t j1, uint32_t* dst, uint32_t lane) {
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t pos = 0;
    for (uint32_t j = j0; j < j1; j += 32) {
        const uint32_t jj = j + lane;
        bool hit = false;
        uint32_t b = 0;
        if (jj < j1) {
            b = sy[jj];
            uint32_t lo = i0, len = i1 - i0;  // i0 + #(sx[i0..i1) < b)
            while (len > 0) {
                const uint32_t half = len >> 1;
                const bool less = sx[lo + half] < b;
                lo = less ? lo + half + 1 : lo;
                len = less ? len - half - 1 : half;
            }
            hit = lo < i1 && sx[lo] == b;
        }
        const uint32_t m = __ballot_sync(kFullMask, hit);
        if (kOut && hit) dst[pos + __popc(m & lt)] = b;
        pos += __popc(m);
    }
    return pos;
}

__device__ __forceinline__ uint32_t lower_bound_smem(const uint32_t* s, uint32_t n, uint32_t v) {
    uint32_t lo = 0, len = n;
    while (len > 0) {
        const uint32_t half = len >> 1;
        const bool less = s[lo + half] < v;
        lo = less ? lo + half + 1 : lo;
        len = less ? len - half - 1 : half;
    }
    return lo;
}

template <bool kOut>
__global__ void __launch_bounds__(kBpBlock, 1) bp_tile_kernel(
    const uint32_t* __restrict__ X, uint64_t nX, const uint32_t* __restrict__ Y, uint64_t nY,
    const uint64_t* __restrict__ split_x, const uint64_t* __restrict__ split_y, uint64_t nTiles,
    unsigned char* __restrict__ ws, uint32_t* __restrict__ unit_count, uint32_t* __restrict__ unit_y,
    uint32_t* __restrict__ scratch, uint64_t* __restrict__ d_count) {
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* ring = smem;
    __shared__ __align__(8) uint64_t full[kBpSlots], ready[kBpSlots], empty[kBpSlots];
    __shared__ BpDesc desc[kBpSlots];
    __shared__ uint64_t s_end[kBpSlots];               // staging lane: ring end (virtual) of each slot's tile
    __shared__ uint32_t s_jb[kBpSlots][kBpWarps + 1];  // Y start of each consumer's range, then ny
    __shared__ volatile uint32_t s_abort;              // the boundary warp gave up: consumers stop
    uint32_t* err = reinterpret_cast<uint32_t*>(ws);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // bitmaps start clear; each consumer clears the words it set after each tile
    for (uint32_t w = tid; w < kBpWarps * kBpWords; w += kBpBlock) smem[kBpRing + w] = 0u;
    if (tid == 0) {
        for (int i = 0; i < kBpSlots; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&ready[i], 1);
            mbar_init(&empty[i], kBpWarps);
        }
        s_abort = 0;
        fence_mbar_init();
    }
    __syncthreads();
    // everything below reads what the split kernel wrote (ticket, splits)
    asm volatile("griddepcontrol.wait;" ::: "memory");

    if (warp == kBpStageWarp) {
        // ------------------------------------------------------- staging --
        if (lane != 0) return;
        uint32_t* ticket = reinterpret_cast<uint32_t*>(ws + 16);
        uint64_t head = 0, released = 0;  // virtual ring offsets
        uint32_t k = 0, k_rel = 0;        // tiles staged / tiles released by every consumer
        auto wait_release = [&]() -> bool {
            const uint32_t sl = k_rel % kBpSlots;
            if (!mbar_wait_bounded(&empty[sl], (k_rel / kBpSlots) & 1u, err, 12, k_rel)) return false;
            released = s_end[sl];
            ++k_rel;
            return true;
        };
        // tickets two tiles ahead, split entries one tile ahead
        uint64_t t = atomicAdd(ticket, 1u), t_next = atomicAdd(ticket, 1u);
        uint64_t x0 = 0, x1 = 0, y0 = 0, y1 = 0;
        if (t < nTiles) {
            x0 = split_x[t];
            x1 = split_x[t + 1];
            y0 = split_y[t];
            y1 = split_y[t + 1];
        }
        bool alive = true;
        for (;;) {
            uint64_t t_after = nTiles, nx0 = 0, nx1 = 0, ny0 = 0, ny1 = 0;
            if (t < nTiles) {
                t_after = atomicAdd(ticket, 1u);
                if (t_next < nTiles) {
                    nx0 = split_x[t_next];
                    nx1 = split_x[t_next + 1];
                    ny0 = split_y[t_next];
                    ny1 = split_y[t_next + 1];
                }
            }
            const uint32_t slot = k % kBpSlots;
            while (alive && k_rel + kBpSlots <= k) alive = wait_release();
            if (!alive) break;
            if (t >= nTiles) {  // end marker: never released, not counted in k
                desc[slot].tile = kEndTile;
                mbar_arrive(&full[slot]);
                break;
            }
            const bool ok = x0 <= x1 && x1 <= nX && x1 - x0 <= kBpS && y0 <= y1 && y1 <= nY && y1 - y0 <= kBpS;
            if (!ok) {
                record_error(err, SI_ERR_INVALID_INPUT, 11, static_cast<uint32_t>(t));
                x0 = x1 = y0 = y1 = 0;
            }
            // 16-byte aligned supersets of the parts: every block copied holds
            // an element of the part, so no byte outside the sets' blocks is read
            const uintptr_t xlo = reinterpret_cast<uintptr_t>(X + x0) & ~uintptr_t(15);
            const uintptr_t ylo = reinterpret_cast<uintptr_t>(Y + y0) & ~uintptr_t(15);
            const uint32_t bytesX =
                x1 > x0 ? static_cast<uint32_t>(((reinterpret_cast<uintptr_t>(X + x1) + 15) & ~uintptr_t(15)) - xlo) : 0u;
            const uint32_t bytesY =
                y1 > y0 ? static_cast<uint32_t>(((reinterpret_cast<uintptr_t>(Y + y1) + 15) & ~uintptr_t(15)) - ylo) : 0u;
            const uint32_t need = (bytesX + bytesY) / 4;
            // a tile never wraps; it is placed once it overlaps no live tile
            const uint64_t phys = head % kBpRing;
            if (phys + need > kBpRing) head += kBpRing - phys;
            while (alive && k_rel < k && head + need - released > kBpRing) alive = wait_release();
            if (!alive) break;
            const uint32_t pos = static_cast<uint32_t>(head % kBpRing);
            head += need;
            s_end[slot] = head;
            BpDesc& d = desc[slot];
            d.tile = static_cast<uint32_t>(t);
            d.y0 = y0;
            d.misX = static_cast<uint32_t>((reinterpret_cast<uintptr_t>(X + x0) & 15u) >> 2);
            d.offX = pos + d.misX;
            d.offY = pos + bytesX / 4 + static_cast<uint32_t>((reinterpret_cast<uintptr_t>(Y + y0) & 15u) >> 2);
            d.nx = static_cast<uint32_t>(x1 - x0);
            d.ny = static_cast<uint32_t>(y1 - y0);
            mbar_arrive_expect_tx(&full[slot], bytesX + bytesY);
            if (bytesX) bulk_g2s(ring + pos, reinterpret_cast<const void*>(xlo), bytesX, &full[slot]);
            if (bytesY) bulk_g2s(ring + pos + bytesX / 4, reinterpret_cast<const void*>(ylo), bytesY, &full[slot]);
            ++k;
            t = t_next;
            t_next = t_after;
            x0 = nx0;
            x1 = nx1;
            y0 = ny0;
            y1 = ny1;
        }
        // the copies in flight land before the CTA may exit: normally every
        // staged tile (k of them, the end marker not counted) is released; if
        // a wait gave up, wait for the copies themselves (bounded)
        while (alive && k_rel < k) alive = wait_release();
        for (uint32_t q = k_rel; q < k; ++q) mbar_wait_bounded(&full[q % kBpSlots], (q / kBpSlots) & 1u, err, 13, q);
        return;
    }

    if (warp == kBpBoundWarp) {
        // ---------------------------------------------------- boundaries --
        // Lane w < 30: the first Y element of consumer w's value range, i.e.
        // #(Y part < its first X element); lane 30: ny.
        for (uint32_t k = 0;; ++k) {
            const uint32_t slot = k % kBpSlots;
            if (!mbar_wait_bounded(&full[slot], (k / kBpSlots) & 1u, err, 15, k)) {
                if (lane == 0) {
                    s_abort = 1u;
                    mbar_arrive(&ready[slot]);
                }
                return;
            }
            const BpDesc d = desc[slot];
            if (d.tile != kEndTile) {
                uint32_t jb = d.ny;
                if (lane < kBpWarps) {
                    const uint32_t i0 = (lane * d.nx) / kBpWarps;
                    if (i0 < d.nx) jb = lower_bound_smem(ring + d.offY, d.ny, ring[d.offX + i0]);
                }
                // sorted sets give nondecreasing boundaries
                const uint32_t prev = __shfl_up_sync(kFullMask, jb, 1);
                if (lane >= 1 && lane <= kBpWarps && prev > jb) record_error(err, SI_ERR_INVALID_INPUT, 18, d.tile);
                if (lane <= kBpWarps) s_jb[slot][lane] = jb;
                if (kOut && lane < kBpWarps) unit_y[static_cast<uint64_t>(d.tile) * kBpWarps + lane] = jb;
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&ready[slot]);
            if (d.tile == kEndTile) return;
        }
    }

    // ------------------------------------------------------- consumers --
    uint32_t* bm = smem + kBpRing + warp * kBpWords;
    uint64_t my_hits = 0;
    for (uint32_t k = 0;; ++k) {
        const uint32_t slot = k % kBpSlots, par = (k / kBpSlots) & 1u;
        if (!mbar_wait_bounded(&ready[slot], par, err, 16, k)) break;
        if (s_abort) break;
        const BpDesc d = desc[slot];
        if (d.tile == kEndTile) break;
        // the boundary warp saw the data land; this wait is already complete
        // and orders this warp's reads after the bulk copies as well
        if (!mbar_wait_bounded(&full[slot], par, err, 17, k)) break;
        const uint32_t i0 = (warp * d.nx) / kBpWarps, i1 = ((warp + 1) * d.nx) / kBpWarps;
        const uint32_t j0 = s_jb[slot][warp], j1 = s_jb[slot][warp + 1];
        uint32_t cnt = 0;
        if (i0 < i1 && j0 < j1) {
            const uint32_t* sx = ring + d.offX;
            const uint32_t* sy = ring + d.offY;
            const uint32_t v0 = sx[i0], vl = sx[i1 - 1], span = vl - v0;
            if (vl < v0 && lane == 0) record_error(err, SI_ERR_INVALID_INPUT, 19, d.tile);
            uint32_t* dst = kOut ? scratch + d.y0 + j0 : nullptr;
            if (span < kBpSpan) {
                bp_build(bm, ring, d, i0, i1, v0, lane);
                __syncwarp();
                cnt = bp_probe<kOut>(bm, sy, j0, j1, v0, span, dst, lane);
                __syncwarp();
                uint4* bm4 = reinterpret_cast<uint4*>(bm);
                for (uint32_t q = lane; q <= (span >> 7); q += 32) bm4[q] = make_uint4(0u, 0u, 0u, 0u);
                __syncwarp();
            } else {
                cnt = bp_search<kOut>(sx, i0, i1, sy, j0, j1, dst, lane);
            }
        }
        if constexpr (kOut) {
            if (lane == 0) unit_count[static_cast<uint64_t>(d.tile) * kBpWarps + warp] = cnt;
        } else {
            my_hits += cnt;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[slot]);
    }
    if constexpr (!kOut) {
        if (lane == 0 && my_hits) atomicAdd(reinterpret_cast<unsigned long long*>(d_count), my_hits);
    }
}

// ----------------------------------------------------------------- K4 --
// Units u = 32 g .. 32 g + 31 (one per lane) hold unit_count[u] hits at
// scratch[split_y[u / 30] + unit_y[u] ...] and go to out[unit_off[u] ...]:
// one contiguous output run.  Each lane finds the unit of output position e
// (the last unit whose run starts at or before e) by a search over the lanes.
constexpr int kCopyUnroll = 8;
__global__ void __launch_bounds__(256) bp_copy_kernel(const uint32_t* __restrict__ unit_count,
                                                      const uint64_t* __restrict__ unit_off,
                                                      const uint32_t* __restrict__ unit_y,
                                                      const uint64_t* __restrict__ split_y, uint64_t nUnits,
                                                      const uint32_t* __restrict__ scratch, uint32_t* __restrict__ out,
                                                      uint64_t out_cap, uint64_t* __restrict__ d_count, uint32_t* err) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t nwarps = static_cast<uint64_t>(gridDim.x) * (blockDim.x / 32);
    const uint64_t ngroups = (nUnits + 31) / 32;
    bool overflow = false;
    for (uint64_t g = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / 32; g < ngroups; g += nwarps) {
        const uint64_t u = g * 32 + lane;
        const bool valid = u < nUnits;
        const uint32_t cnt = valid ? unit_count[u] : 0u;
        const uint64_t off = valid ? unit_off[u] : 0ull;
        const uint64_t src = valid ? split_y[u / kBpWarps] + unit_y[u] : 0ull;
        const uint64_t base = __shfl_sync(kFullMask, off, 0);
        const uint64_t rem = nUnits - 1 - g * 32;
        const uint32_t last = rem < 31 ? static_cast<uint32_t>(rem) : 31u;
        const uint32_t total = static_cast<uint32_t>(__shfl_sync(kFullMask, off + cnt, last) - base);
        // invalid lanes start past the end, so no position selects them
        const uint32_t pre = valid ? static_cast<uint32_t>(off - base) : 0xffffffffu;
        if (valid && u == nUnits - 1) *d_count = off + cnt;
        for (uint32_t e0 = 0; e0 < total; e0 += 32 * kCopyUnroll) {
            uint32_t v[kCopyUnroll];
#pragma unroll
            for (int r = 0; r < kCopyUnroll; ++r) {
                const uint32_t e = e0 + 32 * r + lane;
                uint32_t q = 0;
#pragma unroll
                for (uint32_t s = 16; s; s >>= 1) {
                    const uint32_t p = __shfl_sync(kFullMask, pre, q + s);
                    q = p <= e ? q + s : q;
                }
                const uint64_t sq = __shfl_sync(kFullMask, src, q);
                const uint32_t pq = __shfl_sync(kFullMask, pre, q);
                v[r] = e < total ? __ldg(scratch + sq + (e - pq)) : 0u;
            }
#pragma unroll
            for (int r = 0; r < kCopyUnroll; ++r) {
                const uint32_t e = e0 + 32 * r + lane;
                if (e < total) {
                    if (base + e < out_cap) out[base + e] = v[r];
                    else overflow = true;
                }
            }
        }
    }
    if (overflow) record_error(err, SI_ERR_OUTPUT_OVERFLOW, 9, 0);
}

// Workspace: header (error word, ticket), the split table, the unit tables,
// the scratch array of the hits (as long as Y) and the scan's temporary storage.
constexpr size_t kHeaderBytes = 256;

struct BpLayout {
    uint64_t nTiles = 0, nUnits = 0;
    size_t off_split_x = 0, off_split_y = 0, off_count = 0, off_y = 0, off_off = 0, off_scratch = 0, off_cub = 0,
           cub_bytes = 0, total = 0, total_count_only = 0;
};

BpLayout make_bp_layout(uint64_t nA, uint64_t nB) {
    BpLayout L;
    const uint64_t nX = std::max(nA, nB), nY = std::min(nA, nB);
    L.nTiles = (nX + kBpS - 1) / kBpS + (nY + kBpS - 1) / kBpS + 1;
    L.nUnits = L.nTiles * kBpWarps;
    size_t o = kHeaderBytes;
    L.off_split_x = o; o = align_up(o + (L.nTiles + 1) * 8, 256);
    L.off_split_y = o; o = align_up(o + (L.nTiles + 1) * 8, 256);
    L.total_count_only = o;
    L.off_count = o;   o = align_up(o + L.nUnits * 4, 256);
    L.off_y = o;       o = align_up(o + L.nUnits * 4, 256);
    L.off_off = o;     o = align_up(o + L.nUnits * 8, 256);
    L.off_scratch = o; o = align_up(o + nY * 4, 256);
    // without a device to ask, a bound of 1 MiB
    size_t bytes = 0;
    if (L.nUnits > 0x7fffffffull ||
        cub::DeviceScan::ExclusiveScan(nullptr, bytes, static_cast<const uint32_t*>(nullptr),
                                       static_cast<uint64_t*>(nullptr), cub::Sum(), uint64_t(0),
                                       static_cast<int>(std::min<uint64_t>(L.nUnits, 0x7fffffff))) != cudaSuccess)
        bytes = 1u << 20;
    cudaGetLastError();  // a failed query leaves no sticky error behind
    L.cub_bytes = align_up(bytes, 256);
    L.off_cub = o;
    L.total = o + L.cub_bytes;
    return L;
}

}  // namespace

si_status pivot_split(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB, uint64_t S,
                      uint64_t* split_a, uint64_t* split_b, uint64_t* zero, uint64_t nzero, uint64_t* d_count,
                      cudaStream_t stream) {
    const uint64_t nP = (nA + S - 1) / S + (nB + S - 1) / S;
    const uint64_t warps = std::max<uint64_t>(1, std::max(nP, (nzero + 31) / 32));
    const unsigned grid = static_cast<unsigned>(
        std::min<uint64_t>((warps + 7) / 8, static_cast<uint64_t>(sm_count()) * 16));
    PhaseTimer timer("sisi_split", stream);
    pivot_split_kernel<<<grid, 256, 0, stream>>>(dA, nA, dB, nB, S, split_a, split_b, zero, nzero, d_count);
    SI_LAUNCH_CHECK("pivot_split_kernel");
    return SI_OK;
}

size_t bm_workspace_size(uint64_t nA, uint64_t nB) { return make_bp_layout(nA, nB).total; }

si_status bm_sisi(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB, uint64_t* d_count,
                  uint32_t* d_out, uint64_t out_cap, void* ws, size_t ws_bytes, cudaStream_t stream) {
    const BpLayout L = make_bp_layout(nA, nB);
    if (ws_bytes < (d_out ? L.total : L.total_count_only)) return SI_ERR_WORKSPACE_TOO_SMALL;
    if (L.nTiles > 0xffffffffull / kBpWarps || L.nUnits > 0x7fffffffull) return SI_ERR_INVALID_ARGUMENT;
    unsigned char* w = static_cast<unsigned char*>(ws);
    // the smaller set (Y) indexes the scratch array: a unit has at most as
    // many hits as Y elements
    const bool swap = nA < nB;
    const uint32_t* X = swap ? dB : dA;
    const uint32_t* Y = swap ? dA : dB;
    const uint64_t nX = swap ? nB : nA, nY = swap ? nA : nB;
    uint64_t* split_x = reinterpret_cast<uint64_t*>(w + L.off_split_x);
    uint64_t* split_y = reinterpret_cast<uint64_t*>(w + L.off_split_y);
    si_status st = pivot_split(X, nX, Y, nY, kBpS, split_x, split_y, reinterpret_cast<uint64_t*>(w),
                               kHeaderBytes / 8, d_count, stream);
    if (st != SI_OK) return st;
    uint32_t* unit_count = reinterpret_cast<uint32_t*>(w + L.off_count);
    uint32_t* unit_y = reinterpret_cast<uint32_t*>(w + L.off_y);
    uint64_t* unit_off = reinterpret_cast<uint64_t*>(w + L.off_off);
    uint32_t* scratch = reinterpret_cast<uint32_t*>(w + L.off_scratch);
    auto launch = [&](auto kernel) -> si_status {
        SI_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kBpSmem)));
        int per_sm = 0;
        SI_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBpBlock, kBpSmem));
        if (per_sm < 1) return SI_ERR_UNSUPPORTED;
        const unsigned grid =
            static_cast<unsigned>(std::min<uint64_t>(L.nTiles, static_cast<uint64_t>(sm_count()) * per_sm));
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid);
        cfg.blockDim = dim3(kBpBlock);
        cfg.dynamicSmemBytes = kBpSmem;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const uint64_t nTiles = L.nTiles;
        unsigned char* wp = w;
        uint32_t* uc = d_out ? unit_count : nullptr;
        uint32_t* uy = d_out ? unit_y : nullptr;
        uint32_t* sc = d_out ? scratch : nullptr;
        PhaseTimer timer("sisi_tile", stream);
        SI_CUDA_TRY(cudaLaunchKernelEx(&cfg, kernel, X, nX, Y, nY, static_cast<const uint64_t*>(split_x),
                                       static_cast<const uint64_t*>(split_y), nTiles, wp, uc, uy, sc, d_count));
        return SI_OK;
    };
    if (!d_out) return launch(bp_tile_kernel<false>);
    st = launch(bp_tile_kernel<true>);
    if (st != SI_OK) return st;
    {
        PhaseTimer timer("sisi_scan", stream);
        size_t bytes = L.cub_bytes;
        SI_CUDA_TRY(cub::DeviceScan::ExclusiveScan(w + L.off_cub, bytes, unit_count, unit_off, cub::Sum(),
                                                   uint64_t(0), static_cast<int>(L.nUnits), stream));
    }
    {
        PhaseTimer timer("sisi_copy", stream);
        const uint64_t groups = (L.nUnits + 31) / 32;
        const unsigned grid = static_cast<unsigned>(
            std::max<uint64_t>(1, std::min<uint64_t>((groups + 7) / 8, static_cast<uint64_t>(sm_count()) * 8)));
        bp_copy_kernel<<<grid, 256, 0, stream>>>(unit_count, unit_off, unit_y, split_y, L.nUnits, scratch, d_out,
                                                 out_cap, d_count, reinterpret_cast<uint32_t*>(w));
        SI_LAUNCH_CHECK("bp_copy_kernel");
    }
    return SI_OK;
}

}  // namespace si
