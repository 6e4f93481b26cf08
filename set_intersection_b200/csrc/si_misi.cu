// si_misi.cu -- all pairs of a collection of sorted sets (MISI), one tile
// pair at a time, techniques ip / obs / hi / bitmap.
//
// Replaces the reference's per-technique MISI loops: for every tile pair
// (include/util.hpp:40-52) a host loop launches findDiagonals +
// intersectPath (src/ip.cu:141-177, :207-245), warpBasedOBS / blockBasedOBS
// (src/obs.cu:275-438), warpBasedHI / blockBasedHI (src/hi.cu:295-420) or the
// bitmap_dynamic kernels (src/bitmap_dynamic.cu:240-319), each giving a warp or
// block to one set `a` and looping over its partners `b`.  Same result layout
// (triangular for a self-join tile, quadratic for a cross tile, row stride
// = the reference's numOfSets), different schedule:
//
//  * Every pair is handled by its LARGER set (ties: the A side, then the lower
//    index): the larger set x is staged into shared memory once per work item
//    -- as a bitmap of its values (bitmap), an open-addressing hash table (hi),
//    or as the sorted array itself (obs: binary search; ip: merge) -- and the
//    smaller partners y are streamed from global memory against it.  The work
//    is sum over pairs of min(|a|, |b|) probes instead of |a| + |b|.
//  * Plan on the device: each side's sets are sorted by size, descending
//    (radix sort of (size, index) keys), so the partners of a row form a
//    suffix of the other side's sorted list; prefix sums of the sorted sizes
//    number the partners' elements, and every row's suffix is cut into work
//    items of equal element volume (a large partner may span items).
//  * One persistent launch walks the items with an atomic ticket, largest
//    rows first.  Each warp of the CTA takes an equal slice of the item's
//    partner elements and walks it 32 partners at a time: lane q loads the
//    bounds of partner q's piece (one round trip for 32 partners); pieces under
//    64 elements are probed one per lane, all 32 at once, larger ones by the
//    whole warp in turn with coalesced 16-byte loads.  A partner split between
//    slices or items has its partial counts added atomically.
//  * A set larger than one shared-memory structure (bitmap: value span > 2^20,
//    others: > 16384 / 8192 elements) is processed in chunks of consecutive
//    values; partners are then trimmed to the chunk's value range and the
//    chunk counts added atomically.
#include <algorithm>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "si_device.cuh"
#include "si_internal.h"
#include "si_stream.cuh"

namespace si {
namespace {

constexpr int kMisiThreads = 1024;
constexpr int kMisiWarps = kMisiThreads / 32;
constexpr uint32_t kBitmapBits = 1u << 20;             // bitmap: values per chunk (128 KiB)
constexpr uint32_t kSortedChunk = 16384;               // obs / ip: elements per chunk (64 KiB)
constexpr uint32_t kHashChunk = 8192;                  // hi: elements per chunk
constexpr uint32_t kHashTable = 2 * kHashChunk;        // slots (64 KiB), load factor <= 1/2
constexpr uint32_t kHashBits = 14;
static_assert(kHashTable == (1u << kHashBits), "hash table size");
constexpr uint64_t kMinItemWork = 131072;  // partner elements per work item, at least
constexpr uint32_t kLaneCol = 64;          // partner pieces below this size are probed by one lane each
constexpr uint64_t kMinSlice = 4096;       // partner elements per slice a warp takes, at least
constexpr uint32_t kEmpty = 0xffffffffu;
constexpr size_t kMisiHeader = 256;        // [0..16) error words, [16] u32 ticket

// Partner elements of one work item of a row whose set has `size` elements:
// staging the set (rebuilt for every item of its row) costs at most 1/64 of
// the item's probes.  Measured on the power-law collection (bitmap probe):
// 62.8 ms with items of 4x the set, 43.6 with 16x, 39.1 with 32x, 36.8 with
// 64x: the staging's inserts are shared atomics.
constexpr uint64_t kItemPerElement = 64;
__host__ __device__ inline uint64_t item_unit(uint64_t size) {
    return kItemPerElement * size > kMinItemWork ? kItemPerElement * size : kMinItemWork;
}

__host__ __device__ constexpr size_t misi_smem(int tech) {
    return tech == SI_TECH_BITMAP ? kBitmapBits / 8 : tech == SI_TECH_HI ? kHashTable * 4 : kSortedChunk * 4;
}
__host__ __device__ constexpr int misi_ctas_per_sm(int tech) { return tech == SI_TECH_BITMAP ? 1 : 2; }

__host__ __device__ inline uint64_t tri_idx(uint64_t n, uint64_t i, uint64_t j) {
    return (n * (n - 1) / 2) - (n - i) * ((n - i) - 1) / 2 + j - i - 1;
}

struct MisiLayout {
    uint32_t nA = 0, nB = 0, rows = 0;
    bool self = true;
    size_t off_keys_in = 0, off_keys = 0, off_sizes = 0, off_P = 0, off_cs = 0, off_nseg = 0, off_items = 0,
           off_cub = 0, cub_bytes = 0, total = 0;
};

// Sort key of a set: size descending, then local index ascending.
__host__ __device__ inline uint64_t size_key(uint32_t size, uint32_t local) {
    return (uint64_t(0xffffffffu - size) << 32) | local;
}

MisiLayout misi_layout(si_set_range A, si_set_range B) {
    MisiLayout L;
    L.self = A.start == B.start && A.end == B.end;
    L.nA = A.end - A.start;
    L.nB = L.self ? 0 : B.end - B.start;
    L.rows = L.nA + L.nB;
    const uint64_t n = L.rows;
    size_t o = kMisiHeader;
    L.off_keys_in = o;  o = align_up(o + n * 8, 256);
    L.off_keys = o;     o = align_up(o + n * 8, 256);
    L.off_sizes = o;    o = align_up(o + (n + 2) * 8, 256);  // sorted sizes (u64), per side
    L.off_P = o;        o = align_up(o + (n + 2) * 8, 256);  // prefix sums per side: nA + 1, nB + 1
    L.off_cs = o;       o = align_up(o + n * 4, 256);
    L.off_nseg = o;     o = align_up(o + (n + 1) * 8, 256);
    L.off_items = o;    o = align_up(o + (n + 1) * 8, 256);
    // CUB scratch: the larger of the sort and the scans
    // (without a device to ask, a bound: a second key buffer plus 1 MiB)
    size_t sort_bytes = 0, scan_bytes = 0;
    if (cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, static_cast<const uint64_t*>(nullptr),
                                       static_cast<uint64_t*>(nullptr), static_cast<int>(std::max<uint64_t>(n, 1))) !=
        cudaSuccess)
        sort_bytes = n * 8 + (1u << 20);
    if (cub::DeviceScan::InclusiveSum(nullptr, scan_bytes, static_cast<const uint64_t*>(nullptr),
                                      static_cast<uint64_t*>(nullptr), static_cast<int>(n + 1)) != cudaSuccess)
        scan_bytes = 1u << 20;
    cudaGetLastError();  // a failed query leaves no sticky error behind
    L.cub_bytes = align_up(std::max(sort_bytes, scan_bytes), 256);
    L.off_cub = o;
    o += L.cub_bytes;
    L.total = o;
    return L;
}

// ------------------------------------------------------------------ plan --
__global__ void misi_keys_kernel(const uint64_t* __restrict__ off, uint32_t a_start, uint32_t nA, uint32_t b_start,
                                 uint32_t nB, uint64_t* __restrict__ keys, uint32_t* err) {
    const uint32_t n = nA + nB;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const bool isA = i < nA;
        const uint32_t local = isA ? i : i - nA;
        const uint32_t id = (isA ? a_start : b_start) + local;
        const uint64_t size = off[id + 1] - off[id];
        if (size > 0xffffffffull) record_error(err, SI_ERR_INVALID_INPUT, 40, id);
        keys[i] = size_key(static_cast<uint32_t>(size), local);
    }
}

// sizes[] in sorted order (side A at [0, nA), side B at [nA + 1, nA + 1 + nB))
// with a zero after each side, ready for an inclusive scan into P.
__global__ void misi_sizes_kernel(const uint64_t* __restrict__ keys, uint32_t nA, uint32_t nB,
                                  uint64_t* __restrict__ sizes) {
    const uint32_t n = nA + nB + 2;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint64_t v = 0;
        if (i < nA) v = 0xffffffffull - (keys[i] >> 32);
        else if (i > nA && i < nA + 1 + nB) v = 0xffffffffull - (keys[i - 1] >> 32);
        sizes[i] = v;
    }
}

// First position in the sorted list (sizes descending) whose size is <= s
// (strict: < s).
__device__ __forceinline__ uint32_t first_not_larger(const uint64_t* keys, uint32_t n, uint32_t s, bool strict) {
    uint32_t lo = 0, len = n;
    while (len > 0) {
        const uint32_t half = len >> 1;
        const uint32_t sz = 0xffffffffu - static_cast<uint32_t>(keys[lo + half] >> 32);
        const bool before = strict ? sz >= s : sz > s;
        lo = before ? lo + half + 1 : lo;
        len = before ? len - half - 1 : half;
    }
    return lo;
}

// Per row: where its partners start in the other side's sorted list, and how
// many work items its partners' elements make.  P: exclusive prefix sums.
__global__ void misi_rows_kernel(const uint64_t* __restrict__ keys, uint32_t nA, uint32_t nB, bool self,
                                 const uint64_t* __restrict__ P, uint32_t* __restrict__ cs,
                                 uint64_t* __restrict__ nseg) {
    const uint32_t rows = nA + nB;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r <= rows; r += gridDim.x * blockDim.x) {
        if (r == rows) {
            nseg[r] = 0;
            continue;
        }
        const bool isA = r < nA;
        const uint32_t size = 0xffffffffu - static_cast<uint32_t>(keys[r] >> 32);
        uint32_t c;
        const uint64_t* Pt;
        uint32_t nt;
        if (self) {
            c = r + 1;
            Pt = P;
            nt = nA;
        } else if (isA) {  // partners: B sets no larger than this one
            c = first_not_larger(keys + nA, nB, size, false);
            Pt = P + nA + 1;
            nt = nB;
        } else {           // partners: A sets strictly smaller
            c = first_not_larger(keys, nA, size, true);
            Pt = P;
            nt = nA;
        }
        cs[r] = c;
        const uint64_t work = Pt[nt] - Pt[c];
        const uint64_t unit = item_unit(size);
        nseg[r] = work ? (work + unit - 1) / unit : 0;
    }
}

// ---------------------------------------------------------------- probes --
struct MisiParams {
    const uint32_t* el;
    const uint64_t* off;
    uint32_t a_start, b_start, nA, nB;
    uint32_t self;
    uint64_t stride;
    const uint64_t* keys;   // sorted: side A [0, nA), side B [nA, nA + nB)
    const uint64_t* P;      // side A [0, nA], side B [nA + 1, nA + 1 + nB]
    const uint32_t* cs;
    const uint64_t* items;  // exclusive scan of nseg, rows + 1 entries
    uint32_t* counts;
    uint32_t* ticket;
};

__device__ __forceinline__ uint64_t lower_bound_u64(const uint64_t* x, uint64_t lo, uint64_t hi, uint64_t v) {
    uint64_t len = hi - lo;
    while (len > 0) {
        const uint64_t half = len >> 1;
        const bool c = x[lo + half] < v;
        lo = c ? lo + half + 1 : lo;
        len = c ? len - half - 1 : half;
    }
    return lo;
}

__device__ __forceinline__ uint64_t lower_bound_u32(const uint32_t* x, uint64_t n, uint32_t v) {
    uint64_t lo = 0, len = n;
    while (len > 0) {
        const uint64_t half = len >> 1;
        const bool c = __ldg(x + lo + half) < v;
        lo = c ? lo + half + 1 : lo;
        len = c ? len - half - 1 : half;
    }
    return lo;
}

__device__ __forceinline__ uint32_t hslot(uint32_t v) { return (v * 0x9e3779b1u) >> (32 - kHashBits); }

template <int kTech>
__device__ __forceinline__ uint32_t probe_one(uint32_t v, const uint32_t* sm, uint32_t base, uint32_t span, uint32_t m,
                                              bool has_max) {
    if constexpr (kTech == SI_TECH_BITMAP) {
        const uint32_t o = v - base;
        return o <= span ? (sm[o >> 5] >> (o & 31)) & 1u : 0u;
    } else if constexpr (kTech == SI_TECH_HI) {
        if (v == kEmpty) return has_max ? 1u : 0u;
        uint32_t h = hslot(v), t;
        while ((t = sm[h]) != v && t != kEmpty) h = (h + 1) & (kHashTable - 1);
        return t == v ? 1u : 0u;
    } else {  // obs: branch-free binary search of the staged sorted chunk
        if (m == 0) return 0u;
        uint32_t lo = 0, len = m;
        while (len > 1) {
            const uint32_t half = len >> 1;
            lo = sm[lo + half] <= v ? lo + half : lo;
            len -= half;
        }
        return sm[lo] == v ? 1u : 0u;
    }
}

template <int kTech>
__global__ void __launch_bounds__(kMisiThreads, misi_ctas_per_sm(kTech)) misi_probe_kernel(MisiParams p) {
    extern __shared__ __align__(16) uint32_t sm[];
    __shared__ uint64_t s_item;
    __shared__ unsigned long long s_next;  // the next slice of the item's partner elements
    __shared__ uint32_t s_has_max;
    const int tid = threadIdx.x, lane = tid & 31;
    const uint32_t rows = p.nA + p.nB;
    const uint64_t n_items = p.items[rows];

    for (;;) {
        if (tid == 0) s_item = atomicAdd(p.ticket, 1u);
        __syncthreads();
        const uint64_t item = s_item;
        __syncthreads();  // s_item is rewritten at the next ticket
        if (item >= n_items) break;

        // ---- the item: row r, slice `seg` of the elements of its partners ----
        const uint32_t r = static_cast<uint32_t>(lower_bound_u64(p.items, 0, rows + 1, item + 1) - 1);
        const uint64_t seg = item - p.items[r];
        const bool rowA = r < p.nA;
        const uint32_t x_id = (rowA ? p.a_start : p.b_start) + static_cast<uint32_t>(p.keys[r] & 0xffffffffu);
        const uint64_t* Pt;
        const uint64_t* Kt;
        uint32_t nt, t_start;
        if (p.self || !rowA) {
            Pt = p.P; Kt = p.keys; nt = p.nA; t_start = p.a_start;
        } else {
            Pt = p.P + p.nA + 1; Kt = p.keys + p.nA; nt = p.nB; t_start = p.b_start;
        }
        const uint32_t c_row = p.cs[r];
        const uint64_t x0 = p.off[x_id], nx = p.off[x_id + 1] - x0;
        const uint32_t* x = p.el + x0;
        // partner elements are numbered by Pt (prefix sums of the sorted
        // sizes); this item takes [it_lo, it_hi), and the warps take slices
        // of it from a shared counter (at least 4 per warp), so that a warp
        // whose slices probe faster takes more of them
        const uint64_t unit = item_unit(nx);
        const uint64_t it_lo = Pt[c_row] + seg * unit;
        const uint64_t it_hi = min(it_lo + unit, Pt[nt]);
        const uint64_t span_e = it_hi - it_lo;
        const uint64_t slice = max(kMinSlice, span_e / (4 * kMisiWarps));

        // ---- chunks of x ----
        uint64_t i0 = 0;
        while (i0 < nx) {
            uint64_t i1;
            const uint32_t base = __ldg(x + i0);
            uint32_t span = 0;
            if constexpr (kTech == SI_TECH_BITMAP) {
                const uint64_t top = uint64_t(base) + kBitmapBits - 1;
                i1 = top >= 0xffffffffull ? nx : i0 + lower_bound_u32(x + i0, nx - i0, static_cast<uint32_t>(top) + 1);
                span = __ldg(x + i1 - 1) - base;
                const uint32_t words = (span >> 5) + 1;
                uint4* s4 = reinterpret_cast<uint4*>(sm);
                for (uint32_t w = tid; w < (words + 3) / 4; w += kMisiThreads) s4[w] = make_uint4(0, 0, 0, 0);
                __syncthreads();
                for (uint64_t e = i0 + tid; e < i1; e += kMisiThreads) {
                    const uint32_t o = __ldg(x + e) - base;
                    atomicOr(sm + (o >> 5), 1u << (o & 31));
                }
            } else if constexpr (kTech == SI_TECH_HI) {
                i1 = min(nx, i0 + kHashChunk);
                uint4* s4 = reinterpret_cast<uint4*>(sm);
                for (uint32_t w = tid; w < kHashTable / 4; w += kMisiThreads)
                    s4[w] = make_uint4(kEmpty, kEmpty, kEmpty, kEmpty);
                if (tid == 0) s_has_max = 0;
                __syncthreads();
                for (uint64_t e = i0 + tid; e < i1; e += kMisiThreads) {
                    const uint32_t v = __ldg(x + e);
                    if (v == kEmpty) {
                        s_has_max = 1;
                        continue;
                    }
                    uint32_t h = hslot(v);
                    while (atomicCAS(sm + h, kEmpty, v) != kEmpty) h = (h + 1) & (kHashTable - 1);
                }
            } else {  // obs, ip: the chunk itself
                i1 = min(nx, i0 + kSortedChunk);
                for (uint64_t e = i0 + tid; e < i1; e += kMisiThreads) sm[e - i0] = __ldg(x + e);
            }
            const uint32_t m = static_cast<uint32_t>(i1 - i0);
            const uint32_t vlast = __ldg(x + i1 - 1);
            const bool single = i0 == 0 && i1 == nx;
            if (tid == 0) s_next = it_lo;
            __syncthreads();
            const bool has_max = kTech == SI_TECH_HI ? s_has_max != 0 : false;

            for (;;) {
            // ---- a slice [w_lo, w_hi), 32 partners at a time: lane q takes
            // partner c + q's piece of the slice ----
            unsigned long long w_lo = 0;
            if (lane == 0) w_lo = atomicAdd(&s_next, static_cast<unsigned long long>(slice));
            w_lo = __shfl_sync(kFullMask, w_lo, 0);
            if (w_lo >= it_hi) break;
            const uint64_t w_hi = min(static_cast<uint64_t>(w_lo) + slice, it_hi);
            // the partner holding element w_lo: last c with Pt[c] <= w_lo
            const uint32_t c_first =
                static_cast<uint32_t>(warp_first_true(c_row, nt + 1, [&](uint64_t q) { return Pt[q] > w_lo; }) - 1);
            uint64_t e = w_lo;
            uint32_t c = c_first;
            while (e < w_hi) {
                const uint32_t col = c + lane;
                const uint64_t pc = col <= nt ? Pt[col] : ~0ull;
                const bool valid = col < nt && pc < w_hi;
                uint32_t my_id = 0, n = 0;
                uint64_t y0 = 0, pe = 0;
                bool whole = false;
                if (valid) {
                    const uint64_t pn = Pt[col + 1];
                    const uint64_t ps = max(pc, e);
                    pe = min(pn, w_hi);
                    whole = ps == pc && pe == pn;
                    my_id = t_start + static_cast<uint32_t>(Kt[col] & 0xffffffffu);
                    y0 = p.off[my_id] + (ps - pc);
                    n = static_cast<uint32_t>(pe - ps);
                    if (!single && n) {  // the values of this chunk only
                        const uint32_t* yy = p.el + y0;
                        const uint64_t j0 = lower_bound_u32(yy, n, base);
                        const uint64_t j1 = vlast == 0xffffffffu ? n : lower_bound_u32(yy, n, vlast + 1);
                        y0 += j0;
                        n = j1 > j0 ? static_cast<uint32_t>(j1 - j0) : 0u;
                    }
                }
                const uint32_t nb = __popc(__ballot_sync(kFullMask, valid));  // valid lanes are a prefix
                uint32_t my_hits = 0;
                if constexpr (kTech == SI_TECH_IP) {
                    for (uint32_t q = 0; q < nb; ++q) {
                        const uint32_t ny = __shfl_sync(kFullMask, n, q);
                        const uint32_t* y = p.el + __shfl_sync(kFullMask, y0, q);
                        uint32_t hits = 0;
                        // merge: lane takes y[j0, j1), finds its start in the chunk, walks forward
                        const uint32_t vt = (ny + 31) / 32;
                        const uint32_t j0 = min(ny, lane * vt), j1 = min(ny, j0 + vt);
                        if (j0 < j1) {
                            const uint32_t v0 = __ldg(y + j0);
                            uint32_t qq = 0, len = m;
                            while (len > 0) {
                                const uint32_t half = len >> 1;
                                const bool lt = sm[qq + half] < v0;
                                qq = lt ? qq + half + 1 : qq;
                                len = lt ? len - half - 1 : half;
                            }
                            for (uint32_t j = j0; j < j1 && qq < m; ++j) {
                                const uint32_t v = __ldg(y + j);
                                while (qq < m && sm[qq] < v) ++qq;
                                hits += (qq < m && sm[qq] == v) ? 1u : 0u;
                            }
                        }
                        hits = __reduce_add_sync(kFullMask, hits);
                        if (lane == q) my_hits = hits;
                    }
                } else {
                    // small pieces (< kLaneCol elements): one per lane, all at once
                    if (valid && n < kLaneCol) {
                        const uint32_t* y = p.el + y0;
                        uint32_t j = 0;
                        for (; j + 4 <= n; j += 4) {
                            const uint32_t v0 = __ldg(y + j), v1 = __ldg(y + j + 1), v2 = __ldg(y + j + 2),
                                           v3 = __ldg(y + j + 3);
                            my_hits += probe_one<kTech>(v0, sm, base, span, m, has_max) +
                                       probe_one<kTech>(v1, sm, base, span, m, has_max) +
                                       probe_one<kTech>(v2, sm, base, span, m, has_max) +
                                       probe_one<kTech>(v3, sm, base, span, m, has_max);
                        }
                        for (; j < n; ++j) my_hits += probe_one<kTech>(__ldg(y + j), sm, base, span, m, has_max);
                    }
                    // large pieces: the whole warp, 16-byte loads
                    uint32_t big = __ballot_sync(kFullMask, valid && n >= kLaneCol);
                    while (big) {
                        const int q = __ffs(big) - 1;
                        big &= big - 1;
                        const uint32_t ny = __shfl_sync(kFullMask, n, q);
                        const uint32_t* y = p.el + __shfl_sync(kFullMask, y0, q);
                        const uint32_t head =
                            min(ny, static_cast<uint32_t>((16u - (reinterpret_cast<uintptr_t>(y) & 15u)) & 15u) >> 2);
                        const uint32_t n4 = (ny - head) >> 2;
                        const uint32_t tail0 = head + 4 * n4;
                        uint32_t hits = 0;
                        // head and tail: at most 3 elements each, plain loads
                        if (lane < head) hits += probe_one<kTech>(__ldg(y + lane), sm, base, span, m, has_max);
                        if (lane < ny - tail0)
                            hits += probe_one<kTech>(__ldg(y + tail0 + lane), sm, base, span, m, has_max);
                        const uint4* y4 = reinterpret_cast<const uint4*>(y + head);
                        // kLd 16-byte loads in flight per lane (the bitmap probe is
                        // the cheapest per element, so it keeps the most loads going)
                        constexpr uint32_t kLd = kTech == SI_TECH_BITMAP ? 4 : 2;
                        for (uint32_t i = lane; i < n4; i += 32 * kLd) {
                            uint4 g[kLd];
#pragma unroll
                            for (uint32_t u = 0; u < kLd; ++u)
                                g[u] = i + 32 * u < n4 ? __ldg(y4 + i + 32 * u) : make_uint4(0, 0, 0, 0);
#pragma unroll
                            for (uint32_t u = 0; u < kLd; ++u)
                                if (i + 32 * u < n4)
                                    hits += probe_one<kTech>(g[u].x, sm, base, span, m, has_max) +
                                            probe_one<kTech>(g[u].y, sm, base, span, m, has_max) +
                                            probe_one<kTech>(g[u].z, sm, base, span, m, has_max) +
                                            probe_one<kTech>(g[u].w, sm, base, span, m, has_max);
                        }
                        hits = __reduce_add_sync(kFullMask, hits);
                        if (lane == q) my_hits = hits;
                    }
                }
                if (valid) {
                    uint64_t idx;
                    if (p.self) {
                        const uint32_t a = min(x_id, my_id) - p.a_start, b = max(x_id, my_id) - p.a_start;
                        idx = tri_idx(p.stride, a, b);
                    } else {
                        const uint32_t a = rowA ? x_id : my_id, b = rowA ? my_id : x_id;
                        idx = uint64_t(a - p.a_start) * p.stride + (b - p.b_start);
                    }
                    // a partner split between slices (or x between chunks) is summed atomically
                    if (single && whole) p.counts[idx] = my_hits;
                    else if (my_hits) atomicAdd(p.counts + idx, my_hits);
                }
                e = __shfl_sync(kFullMask, pe, nb - 1);
                c += nb;
            }
            }
            __syncthreads();  // the structure is rebuilt for the next chunk / item
            i0 = i1;
        }
    }
}

}  // namespace

size_t misi_workspace_size(si_set_range A, si_set_range B) { return misi_layout(A, B).total; }

si_status misi_tile(const uint32_t* d_elements, const uint64_t* d_offsets, si_technique t, si_set_range A,
                    si_set_range B, uint64_t stride, uint32_t* d_counts, void* ws, size_t ws_bytes,
                    cudaStream_t stream) {
    const MisiLayout L = misi_layout(A, B);
    if (ws_bytes < L.total) return SI_ERR_WORKSPACE_TOO_SMALL;
    unsigned char* w = static_cast<unsigned char*>(ws);
    uint32_t* err = reinterpret_cast<uint32_t*>(w);
    SI_CUDA_TRY(cudaMemsetAsync(w, 0, kMisiHeader, stream));
    // every count of the tile starts at zero (pairs with an empty set are never visited)
    const uint64_t n_counts = L.self ? (L.nA < 2 ? 0 : tri_idx(stride, L.nA - 2, L.nA - 1) + 1)
                                     : (L.nA && L.nB ? uint64_t(L.nA - 1) * stride + L.nB : 0);
    if (n_counts == 0) return SI_OK;
    SI_CUDA_TRY(cudaMemsetAsync(d_counts, 0, n_counts * 4, stream));

    uint64_t* keys_in = reinterpret_cast<uint64_t*>(w + L.off_keys_in);
    uint64_t* keys = reinterpret_cast<uint64_t*>(w + L.off_keys);
    uint64_t* sizes = reinterpret_cast<uint64_t*>(w + L.off_sizes);
    uint64_t* P = reinterpret_cast<uint64_t*>(w + L.off_P);
    uint32_t* cs = reinterpret_cast<uint32_t*>(w + L.off_cs);
    uint64_t* nseg = reinterpret_cast<uint64_t*>(w + L.off_nseg);
    uint64_t* items = reinterpret_cast<uint64_t*>(w + L.off_items);
    void* cub_tmp = w + L.off_cub;
    const unsigned g = static_cast<unsigned>(std::min<uint64_t>((L.rows + 255) / 256 + 1, uint64_t(sm_count()) * 8));
    {
        PhaseTimer timer("misi_plan", stream);
        misi_keys_kernel<<<g, 256, 0, stream>>>(d_offsets, A.start, L.nA, B.start, L.nB, keys_in, err);
        SI_LAUNCH_CHECK("misi_keys_kernel");
        size_t tmp = L.cub_bytes;
        SI_CUDA_TRY(cub::DeviceRadixSort::SortKeys(cub_tmp, tmp, keys_in, keys, static_cast<int>(L.nA), 0, 64, stream));
        if (L.nB) {
            tmp = L.cub_bytes;
            SI_CUDA_TRY(cub::DeviceRadixSort::SortKeys(cub_tmp, tmp, keys_in + L.nA, keys + L.nA,
                                                       static_cast<int>(L.nB), 0, 64, stream));
        }
        misi_sizes_kernel<<<g, 256, 0, stream>>>(keys, L.nA, L.nB, sizes);
        SI_LAUNCH_CHECK("misi_sizes_kernel");
        // P[i] = sum of sizes[0 .. i) per side: an inclusive scan stored one place on
        SI_CUDA_TRY(cudaMemsetAsync(P, 0, 8, stream));
        tmp = L.cub_bytes;
        SI_CUDA_TRY(cub::DeviceScan::InclusiveSum(cub_tmp, tmp, sizes, P + 1, static_cast<int>(L.nA), stream));
        if (L.nB) {
            SI_CUDA_TRY(cudaMemsetAsync(P + L.nA + 1, 0, 8, stream));
            tmp = L.cub_bytes;
            SI_CUDA_TRY(cub::DeviceScan::InclusiveSum(cub_tmp, tmp, sizes + L.nA + 1, P + L.nA + 2,
                                                      static_cast<int>(L.nB), stream));
        }
        misi_rows_kernel<<<g, 256, 0, stream>>>(keys, L.nA, L.nB, L.self, P, cs, nseg);
        SI_LAUNCH_CHECK("misi_rows_kernel");
        tmp = L.cub_bytes;
        SI_CUDA_TRY(cub::DeviceScan::ExclusiveSum(cub_tmp, tmp, nseg, items, static_cast<int>(L.rows + 1), stream));
    }

    MisiParams prm;
    prm.el = d_elements;
    prm.off = d_offsets;
    prm.a_start = A.start;
    prm.b_start = B.start;
    prm.nA = L.nA;
    prm.nB = L.nB;
    prm.self = L.self;
    prm.stride = stride;
    prm.keys = keys;
    prm.P = P;
    prm.cs = cs;
    prm.items = items;
    prm.counts = d_counts;
    prm.ticket = reinterpret_cast<uint32_t*>(w + 16);

    auto launch = [&](auto kernel, int tech) -> si_status {
        const size_t smem = misi_smem(tech);
        SI_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
        const unsigned grid = static_cast<unsigned>(sm_count() * misi_ctas_per_sm(tech));
        PhaseTimer timer("misi_probe", stream);
        kernel<<<grid, kMisiThreads, smem, stream>>>(prm);
        SI_LAUNCH_CHECK("misi_probe_kernel");
        return SI_OK;
    };
    switch (t) {
        case SI_TECH_IP: return launch(misi_probe_kernel<SI_TECH_IP>, SI_TECH_IP);
        case SI_TECH_OBS: return launch(misi_probe_kernel<SI_TECH_OBS>, SI_TECH_OBS);
        case SI_TECH_HI: return launch(misi_probe_kernel<SI_TECH_HI>, SI_TECH_HI);
        case SI_TECH_BITMAP: return launch(misi_probe_kernel<SI_TECH_BITMAP>, SI_TECH_BITMAP);
        default: return SI_ERR_UNSUPPORTED;
    }
}

}  // namespace si
