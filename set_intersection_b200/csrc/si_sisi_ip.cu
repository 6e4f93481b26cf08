// si_sisi_ip.cu -- intersect-path (ip) for one pair of large sorted sets.
//
// Replaces findDiagonals (include/helpers.cuh:75-166) + intersectPath
// (src/ip.cu:207-245) for the single-instance case.  Same two-level idea --
// split the merge path of (A, B) into CTA tiles, then each thread takes a
// sub-diagonal of its tile and merges serially (include/helpers.cuh:24-61) --
// re-designed for B200:
//
//  * Grid level: instead of one 32-thread warp probe per diagonal per pair,
//    tiles are cut at VALUE pivots.  Every S-th element of A and of B is a
//    pivot (S = 4096); a pivot's exact position in the other set is found with
//    one bounded binary search inside an S-element window that the sample
//    merge identifies.  Consecutive pivots bound a tile to <= S elements of
//    each set, and because a tile boundary is a value, an equal pair is never
//    split across tiles (no "augmentation" atomic, quirk of
//    include/helpers.cuh:121-124).
//  * Staging: each tile's A and B ranges are copied into shared memory by the
//    bulk-copy (TMA) engine, 16-byte aligned middle + <= 3 ragged elements per
//    edge by plain loads; every input byte is read from HBM once.
//  * Thread level: merge-path split per thread in shared memory with one
//    tie rule (A first on ties), then a sentinel-terminated serial merge.
//  * Output: matches are compacted per tile and placed with a decoupled
//    look-back over tile aggregates (single pass); count-only mode instead
//    accumulates tile counts into 256 spread partial sums.
#include <algorithm>

#include "si_device.cuh"
#include "si_internal.h"

namespace si {
namespace {

constexpr uint32_t kS = 4096;                     // pivot (sample) stride
constexpr int kThreads = 256;                     // threads per tile CTA
constexpr int kVTMax = (2 * kS) / kThreads;       // merge steps per thread, max
constexpr int kSlots = kVTMax / 2 + 1;            // match slots per thread
constexpr int kBufElems = kS + 8;                 // per-set stage buffer (+align, sentinel)
constexpr size_t kSmemBytes = (2 * kBufElems + kThreads * kSlots) * sizeof(uint32_t);
constexpr int kPartials = 256;

constexpr uint64_t kFlagAgg = 1ull << 62;
constexpr uint64_t kFlagInc = 2ull << 62;
constexpr uint64_t kValMask = (1ull << 62) - 1;
constexpr uint64_t kPoison = ~0ull;

// Workspace layout.  Offsets in bytes from the workspace base.
struct Layout {
    uint64_t nSA = 0, nSB = 0, nTiles = 0;
    size_t off_status = 0, off_split_a = 0, off_split_b = 0, off_sa = 0, off_sb = 0, total = 0;
};
// Header: [0] u32 error word, [4] u32 tile ticket, [8] u32 tiles done,
// [64, 64 + 8*kPartials) u64 partial counts.
constexpr size_t kOffTicket = 4, kOffDone = 8, kOffPartials = 64;

Layout make_layout(uint64_t nA, uint64_t nB) {
    Layout L;
    L.nSA = (nA + kS - 1) / kS;
    L.nSB = (nB + kS - 1) / kS;
    L.nTiles = L.nSA + L.nSB + 1;
    size_t o = align_up(kOffPartials + 8 * kPartials, 256);
    L.off_status = o;
    o = align_up(o + L.nTiles * 8, 256);
    L.off_split_a = o;
    o = align_up(o + (L.nTiles + 1) * 8, 256);
    L.off_split_b = o;
    o = align_up(o + (L.nTiles + 1) * 8, 256);
    L.off_sa = o;
    o = align_up(o + L.nSA * 4, 256);
    L.off_sb = o;
    o = align_up(o + L.nSB * 4, 256);
    L.total = o;
    return L;
}

__device__ __forceinline__ uint64_t lower_bound_g(const uint32_t* __restrict__ x, uint64_t n, uint32_t v) {
    uint64_t lo = 0, hi = n;  // #(x < v)
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if (__ldg(x + mid) < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ uint64_t upper_bound_g(const uint32_t* __restrict__ x, uint64_t n, uint32_t v) {
    uint64_t lo = 0, hi = n;  // #(x <= v)
    while (lo < hi) {
        uint64_t mid = (lo + hi) >> 1;
        if (__ldg(x + mid) <= v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// K1: gather the pivot samples, clear the header + tile status words, poison
// the split table (so a hole left by unsorted input is detected, not used).
__global__ void ip_prepare_kernel(const uint32_t* __restrict__ A, const uint32_t* __restrict__ B,
                                  uint32_t* __restrict__ sa, uint64_t nSA, uint32_t* __restrict__ sb, uint64_t nSB,
                                  uint64_t* __restrict__ zero, uint64_t nzero, uint64_t* __restrict__ split_a,
                                  uint64_t* __restrict__ split_b, uint64_t nsplit) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t t0 = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    for (uint64_t k = t0; k < nSA; k += stride) sa[k] = __ldg(A + k * kS);
    for (uint64_t k = t0; k < nSB; k += stride) sb[k] = __ldg(B + k * kS);
    for (uint64_t k = t0; k < nzero; k += stride) zero[k] = 0;
    for (uint64_t k = t0; k < nsplit; k += stride) {
        split_a[k] = kPoison;
        split_b[k] = kPoison;
    }
}

// K2: one thread per pivot.  Pivot p (A sample k or B sample j) gets its rank
// u in the merged sample order (ties: A sample first) and its exact split
// (#A < v, #B < v), stored at split[u + 1].  split[0] = (0,0) and
// split[nSA + nSB + 1] = (nA, nB) close the table.
__global__ void ip_split_kernel(const uint32_t* __restrict__ A, uint64_t nA, const uint32_t* __restrict__ B,
                                uint64_t nB, const uint32_t* __restrict__ sa, uint64_t nSA,
                                const uint32_t* __restrict__ sb, uint64_t nSB, uint64_t* __restrict__ split_a,
                                uint64_t* __restrict__ split_b) {
    const uint64_t p = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t nP = nSA + nSB;
    if (p == 0) {
        split_a[0] = 0;
        split_b[0] = 0;
        split_a[nP + 1] = nA;
        split_b[nP + 1] = nB;
    }
    if (p >= nP) return;
    if (p < nSA) {
        const uint64_t k = p;
        const uint32_t v = __ldg(sa + k);
        const uint64_t j = lower_bound_g(sb, nSB, v);  // B samples < v
        uint64_t lbB = 0;
        if (j > 0) {  // B[(j-1)S] < v <= B[jS]  =>  #B<v in ((j-1)S, jS]
            const uint64_t lo = (j - 1) * kS + 1;
            const uint64_t hi = min(j * kS, nB);
            lbB = lo + lower_bound_g(B + lo, hi > lo ? hi - lo : 0, v);
        }
        split_a[k + j + 1] = k * kS;
        split_b[k + j + 1] = lbB;
    } else {
        const uint64_t j = p - nSA;
        const uint32_t v = __ldg(sb + j);
        const uint64_t i = upper_bound_g(sa, nSA, v);  // A samples <= v
        uint64_t lbA = 0;
        if (i > 0) {
            if (__ldg(sa + i - 1) == v) {
                lbA = (i - 1) * kS;
            } else {  // A[(i-1)S] < v < A[iS]
                const uint64_t lo = (i - 1) * kS + 1;
                const uint64_t hi = min(i * kS, nA);
                lbA = lo + lower_bound_g(A + lo, hi > lo ? hi - lo : 0, v);
            }
        }
        split_a[i + j + 1] = lbA;
        split_b[i + j + 1] = j * kS;
    }
}

// K3: one CTA per tile, tiles taken in ticket order (so the look-back only
// ever waits on CTAs that are already running).
template <bool kOut>
__global__ void __launch_bounds__(kThreads) ip_tile_kernel(
    const uint32_t* __restrict__ A, uint64_t nA, const uint32_t* __restrict__ B, uint64_t nB,
    const uint64_t* __restrict__ split_a, const uint64_t* __restrict__ split_b, uint64_t nTiles,
    unsigned char* __restrict__ ws, uint64_t* __restrict__ status, uint32_t* __restrict__ out, uint64_t out_cap,
    uint64_t* __restrict__ d_count) {
    extern __shared__ __align__(16) uint32_t smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[kThreads / 32];
    __shared__ uint64_t s_prefix;
    __shared__ uint32_t s_last;

    uint32_t* err = reinterpret_cast<uint32_t*>(ws);
    uint32_t* ticket = reinterpret_cast<uint32_t*>(ws + kOffTicket);
    uint32_t* done = reinterpret_cast<uint32_t*>(ws + kOffDone);
    uint64_t* partials = reinterpret_cast<uint64_t*>(ws + kOffPartials);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint32_t* bufA = smem;
    uint32_t* bufB = smem + kBufElems;
    uint32_t* slots = smem + 2 * kBufElems;

    if (tid == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
        s_tile = atomicAdd(ticket, 1u);
    }
    __syncthreads();
    const uint64_t t = s_tile;

    uint64_t a0 = split_a[t], a1 = split_a[t + 1], b0 = split_b[t], b1 = split_b[t + 1];
    const bool ok = a0 <= a1 && a1 <= nA && a1 - a0 <= kS && b0 <= b1 && b1 <= nB && b1 - b0 <= kS;
    if (!ok) {
        if (tid == 0) record_error(err, SI_ERR_INVALID_INPUT);
        a0 = a1 = b0 = b1 = 0;
    }
    const int na = static_cast<int>(a1 - a0), nb = static_cast<int>(b1 - b0);
    const uint32_t* gA = A + a0;
    const uint32_t* gB = B + b0;
    const StagePlan pa = plan_stage(gA, na, bufA);
    const StagePlan pb = plan_stage(gB, nb, bufB);
    if (tid == 0) {
        mbar_arrive_expect_tx(&bar, static_cast<uint32_t>(pa.body + pb.body) * 4u);
        issue_stage(pa, gA, &bar);
        issue_stage(pb, gB, &bar);
    }
    if (tid < 6) edge_stage(pa, gA, tid);
    else if (tid >= 32 && tid < 38) edge_stage(pb, gB, tid - 32);
    else if (tid == 64) pa.dst[na] = 0xffffffffu;  // sentinels
    else if (tid == 65) pb.dst[nb] = 0xffffffffu;
    mbar_wait_bounded(&bar, 0, err);
    __syncthreads();

    // ---- thread-level merge path ----
    const uint32_t* sA = pa.dst;
    const uint32_t* sB = pb.dst;
    const int L = na + nb;
    const int VT = (L + kThreads - 1) / kThreads;
    const int d0 = min(tid * VT, L), d1 = min(d0 + VT, L);
    int lo = max(0, d0 - nb), hi = min(d0, na);
    while (lo < hi) {  // A first on ties: A[mid] precedes B[d0-1-mid] iff A[mid] <= B[d0-1-mid]
        const int mid = (lo + hi) >> 1;
        if (sA[mid] <= sB[d0 - 1 - mid]) lo = mid + 1; else hi = mid;
    }
    int i = lo, j = d0 - lo;
    uint32_t* my = slots + tid * kSlots;
    int cnt = 0;
    if (t + 1 < nTiles) {
        // Every value of a non-final tile is below the next pivot, hence below
        // 0xffffffff: the sentinels terminate each side without bounds checks.
        uint32_t a = sA[i], b = sB[j];
        for (int s = d0; s < d1; ++s) {
            if (a == b) {
                my[cnt < kSlots ? cnt : kSlots - 1] = a;
                ++cnt;
            }
            if (a <= b) a = sA[++i]; else b = sB[++j];
        }
    } else {
        // Final tile: may hold the value 0xffffffff, so check bounds explicitly.
        for (int s = d0; s < d1; ++s) {
            const bool aOk = i < na, bOk = j < nb;
            const uint32_t a = aOk ? sA[i] : 0u, b = bOk ? sB[j] : 0u;
            const bool takeA = aOk && (!bOk || a <= b);
            if (takeA && bOk && a == b) {
                my[cnt < kSlots ? cnt : kSlots - 1] = a;
                ++cnt;
            }
            if (takeA) ++i; else ++j;
        }
    }
    if (cnt > kSlots) {  // only possible for input that is not strictly increasing
        record_error(err, SI_ERR_INVALID_INPUT);
        cnt = kSlots;
    }

    // ---- block scan of per-thread match counts ----
    const uint32_t incl = warp_inclusive_scan(static_cast<uint32_t>(cnt));
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t v = lane < kThreads / 32 ? s_warp[lane] : 0u;
        v = warp_inclusive_scan(v);
        if (lane < kThreads / 32) s_warp[lane] = v;
    }
    __syncthreads();
    const uint32_t excl = incl - static_cast<uint32_t>(cnt) + (warp ? s_warp[warp - 1] : 0u);
    const uint32_t tile_count = s_warp[kThreads / 32 - 1];

    if constexpr (!kOut) {
        if (tid == 0) {
            atomicAdd(reinterpret_cast<unsigned long long*>(partials + (t & (kPartials - 1))),
                      static_cast<unsigned long long>(tile_count));
            __threadfence();
            s_last = (atomicAdd(done, 1u) == nTiles - 1) ? 1u : 0u;
        }
        __syncthreads();
        if (s_last) {
            __threadfence();
            uint64_t v = 0;
            for (int x = tid; x < kPartials; x += kThreads) v += ld_acquire_u64(partials + x);
            v = warp_sum_u64(v);
            __shared__ uint64_t s_sum[kThreads / 32];
            if (lane == 0) s_sum[warp] = v;
            __syncthreads();
            if (tid == 0) {
                uint64_t total = 0;
                for (int w = 0; w < kThreads / 32; ++w) total += s_sum[w];
                *d_count = total;
            }
        }
        return;
    } else {
        // Compact this tile's matches into the (now free) A stage buffer.
        uint32_t* comp = bufA;
        for (int c = 0; c < cnt; ++c) comp[excl + c] = my[c];

        if (warp == 0) {
            uint64_t prefix = 0;
            if (t == 0) {
                if (lane == 0) st_release_u64(status, kFlagInc | tile_count);
            } else {
                if (lane == 0) st_release_u64(status + t, kFlagAgg | tile_count);
                int64_t p = static_cast<int64_t>(t) - 1 - lane;
                bool gave_up = false;
                while (true) {
                    uint64_t s = p >= 0 ? ld_acquire_u64(status + p) : kFlagInc;
                    uint32_t spins = 0;
                    while (__any_sync(kFullMask, (s >> 62) == 0)) {
                        if ((s >> 62) == 0) {
                            __nanosleep(64);
                            s = ld_acquire_u64(status + p);
                        }
                        if (++spins > kSpinLimit) { gave_up = true; break; }
                    }
                    if (__any_sync(kFullMask, gave_up)) {
                        if (lane == 0) record_error(err, SI_ERR_TIMEOUT);
                        break;
                    }
                    const uint32_t inc_mask = __ballot_sync(kFullMask, (s >> 62) == 2);
                    uint64_t v = s & kValMask;
                    if (inc_mask) {
                        const int first = __ffs(inc_mask) - 1;
                        prefix += warp_sum_u64(lane <= first ? v : 0ull);
                        break;
                    }
                    prefix += warp_sum_u64(v);
                    p -= 32;
                }
                if (lane == 0) st_release_u64(status + t, kFlagInc | ((prefix + tile_count) & kValMask));
            }
            if (lane == 0) s_prefix = prefix;
        }
        __syncthreads();
        const uint64_t base = s_prefix;
        bool overflow = false;
        for (uint32_t x = tid; x < tile_count; x += kThreads) {
            const uint64_t pos = base + x;
            if (pos < out_cap) out[pos] = comp[x];
            else overflow = true;
        }
        if (overflow) record_error(err, SI_ERR_OUTPUT_OVERFLOW);
        if (tid == 0 && t + 1 == nTiles) *d_count = base + tile_count;
    }
}

}  // namespace

size_t ip_workspace_size(uint64_t nA, uint64_t nB) { return make_layout(nA, nB).total; }

si_status ip_sisi(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB, uint64_t* d_count,
                  uint32_t* d_out, uint64_t out_cap, void* ws, size_t ws_bytes, cudaStream_t stream) {
    const Layout L = make_layout(nA, nB);
    if (ws_bytes < L.total) return SI_ERR_WORKSPACE_TOO_SMALL;
    if (L.nTiles > 0x7fffffffull) return SI_ERR_INVALID_ARGUMENT;
    unsigned char* w = static_cast<unsigned char*>(ws);
    uint32_t* sa = reinterpret_cast<uint32_t*>(w + L.off_sa);
    uint32_t* sb = reinterpret_cast<uint32_t*>(w + L.off_sb);
    uint64_t* split_a = reinterpret_cast<uint64_t*>(w + L.off_split_a);
    uint64_t* split_b = reinterpret_cast<uint64_t*>(w + L.off_split_b);
    uint64_t* status = reinterpret_cast<uint64_t*>(w + L.off_status);

    const uint64_t nzero = L.off_split_a / 8;
    const uint64_t work1 = std::max(std::max(L.nSA, L.nSB), std::max(nzero, L.nTiles + 1));
    const unsigned grid1 =
        static_cast<unsigned>(std::min<uint64_t>((work1 + 255) / 256, static_cast<uint64_t>(sm_count()) * 8));
    {
    PhaseTimer timer("ip_prepare", stream);
    ip_prepare_kernel<<<grid1, 256, 0, stream>>>(dA, dB, sa, L.nSA, sb, L.nSB, reinterpret_cast<uint64_t*>(w), nzero,
                                                 split_a, split_b, L.nTiles + 1);
    SI_LAUNCH_CHECK("ip_prepare_kernel");
    }

    const uint64_t nP = L.nSA + L.nSB;
    const unsigned grid2 = static_cast<unsigned>(std::max<uint64_t>(1, (nP + 255) / 256));
    {
    PhaseTimer timer("ip_split", stream);
    ip_split_kernel<<<grid2, 256, 0, stream>>>(dA, nA, dB, nB, sa, L.nSA, sb, L.nSB, split_a, split_b);
    SI_LAUNCH_CHECK("ip_split_kernel");
    }

    SI_CUDA_TRY(cudaFuncSetAttribute(ip_tile_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(kSmemBytes)));
    SI_CUDA_TRY(cudaFuncSetAttribute(ip_tile_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(kSmemBytes)));
    PhaseTimer timer("ip_tile", stream);
    if (d_out) {
        ip_tile_kernel<true><<<static_cast<unsigned>(L.nTiles), kThreads, kSmemBytes, stream>>>(
            dA, nA, dB, nB, split_a, split_b, L.nTiles, w, status, d_out, out_cap, d_count);
    } else {
        ip_tile_kernel<false><<<static_cast<unsigned>(L.nTiles), kThreads, kSmemBytes, stream>>>(
            dA, nA, dB, nB, split_a, split_b, L.nTiles, w, status, nullptr, 0, d_count);
    }
    SI_LAUNCH_CHECK("ip_tile_kernel");
    return SI_OK;
}

}  // namespace si
