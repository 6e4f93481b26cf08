// si_sisi_ip.cu -- intersect-path (ip) for one pair of large sorted sets.
//
// Replaces findDiagonals (include/helpers.cuh:75-166) + intersectPath
// (src/ip.cu:207-245) for the single-instance case.  Same two-level idea --
// split the merge path of (A, B) into CTA tiles, then each thread takes a
// sub-diagonal of its tile and merges serially (include/helpers.cuh:24-61) --
// re-designed for B200:
//
//  * Grid level: instead of one 32-thread warp probe per diagonal per pair,
//    tiles are cut at VALUE pivots (pivot_split, si_sisi_bitmap.cu).  Every
//    S-th element of A and of B is a pivot (S = 6144); a pivot's rank in the
//    merged pivot order and its exact position in the other set are found by
//    warp-cooperative searches.  Consecutive pivots bound a tile to <= S
//    elements of each set, and because a tile boundary is a value, an equal
//    pair is never split across tiles (no "augmentation" atomic, quirk of
//    include/helpers.cuh:121-124).
//  * Staging: each tile's A and B ranges are copied into shared memory by the
//    bulk-copy (TMA) engine as their 16-byte aligned supersets (every block
//    copied holds an element of the range); every input byte is read from HBM
//    once.
//  * Thread level: merge-path split per thread in shared memory with one
//    tie rule (A first on ties), then a sentinel-terminated serial merge.
//  * Output: matches are compacted per tile and placed with a decoupled
//    look-back over tile aggregates (single pass); count-only mode instead
//    accumulates tile counts into 256 spread partial sums.
//
// Techniques bitmap (and auto for pairs of similar size) and hi run the stream
// engine of si_sisi_bitmap.cu, which also holds the pivot split.
#include <algorithm>

#include "si_device.cuh"
#include "si_internal.h"

namespace si {
namespace {

constexpr uint32_t kS = 6144;  // pivot (sample) stride: a tile holds at most this many elements of each set
constexpr int kPartials = 256;

constexpr uint64_t kFlagAgg = 1ull << 62;
constexpr uint64_t kFlagInc = 2ull << 62;
constexpr uint64_t kValMask = (1ull << 62) - 1;

// Workspace layout.  Offsets in bytes from the workspace base.
struct Layout {
    uint64_t nTiles = 0;
    size_t off_status = 0, off_split_a = 0, off_split_b = 0, off_samples = 0, total = 0;
};
// Header: [0] u32 error word, [4] u32 error site, [8] u32 error detail,
// [12] u32 sites that gave up, [16] u32 group ticket,
// [64, 64 + 8*kPartials) u64 partial counts.
constexpr size_t kOffTicket = 16, kOffPartials = 64;

Layout make_layout(uint64_t nA, uint64_t nB, uint64_t S) {
    Layout L;
    L.nTiles = (nA + S - 1) / S + (nB + S - 1) / S + 1;
    size_t o = align_up(kOffPartials + 8 * kPartials, 256);
    L.off_status = o;
    o = align_up(o + L.nTiles * 8, 256);
    L.off_split_a = o;
    o = align_up(o + (L.nTiles + 1) * 8, 256);
    L.off_split_b = o;
    o = align_up(o + (L.nTiles + 1) * 8, 256);
    L.off_samples = o;
    o += pivot_samples_bytes(nA, nB, S);
    L.total = o;
    return L;
}

// K3: persistent, warp-specialised tile pipeline.
//
//   warps 0..8  consumers: intersect one tile at a time out of the input ring
//   warp  9     producer:  takes its groups of tiles in order, reads their
//                          splits, stages each tile's A and B ranges into the
//                          input ring with the bulk-copy engine
//   warp 10     output:    per tile, the tile's global output offset (a
//                          decoupled look-back once per group, then a running
//                          sum), then copies the tile's matches from the
//                          output ring to global memory
//
// Input ring: a variable-size, in-order circular buffer (a tile takes about
// |A_t| + |B_t| elements); descriptors pass through kSlots full/empty
// mbarrier pairs.  Every consumer warp arrives on a tile's empty barrier when
// done with it; the producer learns which ring space is free from those
// barriers, in tile order.  With element output, consumers write a tile's
// matches into an output ring (power-of-two, indexed modulo its size, so every
// consumer thread tracks its head without a broadcast) and release the input
// tile at once; the output warp places them once the tile's offset is known.
// Offsets therefore never hold up merging.  Groups of
// kGroup consecutive tiles are handed out by a ticket counter, so a
// look-back only ever waits on tiles owned by CTAs that are already running
// (the launch is also cooperative: every CTA is resident).
constexpr int kConsumerWarps = 9;  // 288 threads: odd VT of the largest tile stays <= 31
constexpr int kConsumers = kConsumerWarps * 32;
constexpr int kProducerWarp = kConsumerWarps;
constexpr int kOutputWarp = kConsumerWarps + 1;
constexpr int kBlock = (kConsumerWarps + 2) * 32;
constexpr int kCtasPerSm = 2;
constexpr int kSlots = 8;
constexpr int kOutQ = 16;                    // output descriptors in flight
constexpr int kGroup = 4;                    // consecutive tiles per scheduling unit (one look-back each)
constexpr uint32_t kInRing = 18432;          // u32: 72 KiB, about three average tiles
constexpr uint32_t kOutRing = 8192;          // u32: 32 KiB, a power of two
// Shared memory: input ring and output ring, 104 KiB: two CTAs per SM.
constexpr size_t kTileSmem = size_t(kInRing + kOutRing) * sizeof(uint32_t);
static_assert((kOutRing & (kOutRing - 1)) == 0, "output ring is indexed modulo its size");
static_assert(kS <= kOutRing, "one tile's matches must fit the output ring");
constexpr uint32_t kEndTile = 0xffffffffu;
constexpr uint32_t kConsumerBar = 1;  // named barrier id of the consumer warps

static_assert(2 * (kS + 8) + 16 <= kInRing, "a tile's aligned superset must fit the input ring");
static_assert((((2 * kS + kConsumers - 1) / kConsumers) | 1) <= 63, "per-thread match mask is 64 bits");
static_assert(kGroup + 1 <= 32, "a group's split entries are held one per lane");

struct InDesc {
    uint32_t tile;
    uint32_t offA, offB;  // ring offsets of element 0 of the staged A / B ranges
    int na, nb;
    uint32_t fast;        // both successor elements staged: sentinel-terminated merge
};

constexpr int kLookBackPerLane = 4;  // status words per lane per round trip
__device__ __forceinline__ uint64_t look_back(uint64_t* status, uint64_t t, uint32_t* err) {
    // Warp-wide; returns the exclusive prefix of tile t (t > 0).  Flag and
    // value share one 64-bit word, so relaxed accesses suffice.  Each round
    // trip reads the 128 nearest unvisited predecessors, lane l holding
    // tiles base - 4l - 1 ... base - 4l - 4.
    const int lane = threadIdx.x & 31;
    uint64_t prefix = 0;
    int64_t base = static_cast<int64_t>(t);
    while (true) {
        uint64_t s[kLookBackPerLane];
        WaitBudget budget;
        bool gave_up = false;
        while (true) {
            // ready when every status nearer than the nearest inclusive one
            // in the window is published (those beyond it do not matter)
            int first_inc = kLookBackPerLane, first_pending = kLookBackPerLane;
#pragma unroll
            for (int q = kLookBackPerLane - 1; q >= 0; --q) {
                const int64_t p = base - 1 - lane * kLookBackPerLane - q;
                s[q] = p >= 0 ? ld_relaxed_u64(status + p) : kFlagInc;
                if ((s[q] >> 62) == 2) first_inc = q;
                if ((s[q] >> 62) == 0) first_pending = q;
            }
            const uint32_t inc_lanes = __ballot_sync(kFullMask, first_inc < kLookBackPerLane);
            const int inc_lane = inc_lanes ? __ffs(inc_lanes) - 1 : 32;
            const int inc_q = __shfl_sync(kFullMask, first_inc, inc_lane & 31);
            // a pending status nearer than (inc_lane, inc_q) blocks
            const bool blocks = first_pending < kLookBackPerLane &&
                                (lane < inc_lane || (lane == inc_lane && first_pending < inc_q));
            if (!__any_sync(kFullMask, blocks)) break;
            if (__any_sync(kFullMask, budget.expired())) {  // warp-uniform exit
                gave_up = true;
                break;
            }
            __nanosleep(32);
        }
        if (gave_up) {
            if (lane == 0) record_error(err, SI_ERR_TIMEOUT, 1, static_cast<uint32_t>(t));
            return prefix;
        }
        // nearest inclusive status in this window: lane-major, then q
        int first_q = kLookBackPerLane;
#pragma unroll
        for (int q = kLookBackPerLane - 1; q >= 0; --q)
            if ((s[q] >> 62) == 2) first_q = q;
        const uint32_t inc_mask = __ballot_sync(kFullMask, first_q < kLookBackPerLane);
        uint64_t v = 0;
        if (inc_mask) {
            const int first_lane = __ffs(inc_mask) - 1;
#pragma unroll
            for (int q = 0; q < kLookBackPerLane; ++q) {
                const bool take = lane < first_lane || (lane == first_lane && q <= first_q);
                v += take ? (s[q] & kValMask) : 0ull;
            }
            return prefix + warp_sum_u64(v);
        }
#pragma unroll
        for (int q = 0; q < kLookBackPerLane; ++q) v += s[q] & kValMask;
        prefix += warp_sum_u64(v);
        base -= 32 * kLookBackPerLane;
    }
}

// ---------------------------------------------------------------------------
// Per-tile inner algorithms.  Each consumer thread ends with the matches it
// owns as a bit mask over a contiguous run of one staged set: the matched
// values are src[start + x] for every set bit x, in ascending order, and the
// runs of consecutive threads are consecutive.
// (kBitmapProbe and kHashProbe select the stream engine of si_sisi_bitmap.cu,
// with window bitmaps or window hash tables.)
enum Inner { kMergePath = 0, kBitmapProbe = 1, kHashProbe = 2 };

struct ThreadMatches {
    const uint32_t* src;
    int start;
    uint64_t mask;
};

// Merge path (the reference's intersect-path, include/helpers.cuh:24-61): the
// thread takes diagonals [d0, d0 + VT) of the tile's merge of A and B, finds
// its split with a branch-free binary search (A first on ties) and merges
// serially; a match is recorded when an A element is consumed while the head
// of B equals it.
__device__ __forceinline__ ThreadMatches merge_inner(const uint32_t* sA, int na, const uint32_t* sB, int nb,
                                                     bool fast, int tid) {
    const int L = na + nb;
    // Odd steps per thread: consecutive threads then start VT/2 (a non-integer)
    // words apart in each set, which spreads their shared loads over the banks.
    const int VT = ((L + kConsumers - 1) / kConsumers) | 1;
    const int d0 = min(tid * VT, L), d1 = min(d0 + VT, L);
    int lo = max(0, d0 - nb), len = min(d0, na) - lo;
    while (len > 0) {
        const int half = len >> 1, mid = lo + half;
        const bool c = sA[mid] <= sB[d0 - 1 - mid];
        lo = c ? mid + 1 : lo;
        len = c ? len - half - 1 : half;
    }
    const int i0 = lo;
    uint64_t mask = 0;  // bit x: A element i0 + x is in B
    if (fast) {
        // sA[na] / sB[nb] are the successor elements of the ranges, both at or
        // above the next pivot and so above every value of the tile: they stop
        // each side without bounds checks.  One shared load per step, through
        // 32-bit shared-window byte addresses.
        uint32_t pa = smem_addr(sA + i0), pb = smem_addr(sB + (d0 - i0));
        uint32_t a = lds_u32(pa), b = lds_u32(pb), ka = 0;
        const int steps = d1 - d0;
#pragma unroll 4
        for (int s = 0; s < steps; ++s) {
            const bool takeA = a <= b;
            mask |= static_cast<uint64_t>(a == b) << ka;
            ka += takeA ? 1u : 0u;
            pa += takeA ? 4u : 0u;
            pb += takeA ? 0u : 4u;
            const uint32_t v = lds_u32(takeA ? pa : pb);
            a = takeA ? v : a;
            b = takeA ? b : v;
        }
    } else {
        int i = i0, j = d0 - i0;
        for (int s = d0; s < d1; ++s) {
            const bool aOk = i < na, bOk = j < nb;
            const uint32_t a = aOk ? sA[i] : 0u, b = bOk ? sB[j] : 0u;
            const bool takeA = aOk && (!bOk || a <= b);
            if (takeA && bOk && a == b) mask |= 1ull << (i - i0);
            if (takeA) ++i; else ++j;
        }
    }
    return {sA, i0, mask};
}

template <bool kOut>
__global__ void __launch_bounds__(kBlock, kCtasPerSm) ip_tile_kernel(
    const uint32_t* __restrict__ A, uint64_t nA, const uint32_t* __restrict__ B, uint64_t nB,
    const uint64_t* __restrict__ split_a, const uint64_t* __restrict__ split_b, uint64_t nTiles,
    unsigned char* __restrict__ ws, uint64_t* __restrict__ status, uint32_t* __restrict__ out, uint64_t out_cap,
    uint64_t* __restrict__ d_count) {
    extern __shared__ __align__(16) uint32_t smem[];
    uint32_t* in_ring = smem;
    constexpr uint32_t kRing = kInRing;
    constexpr uint64_t kTileMax = kS;
    uint32_t* out_ring = smem + kRing;
    __shared__ __align__(8) uint64_t full[kSlots], empty[kSlots], ofull[kOutQ], oempty[kOutQ];
    __shared__ __align__(8) uint64_t s_released_out;  // output ring: virtual offset written out so far
    __shared__ uint32_t s_otile[kOutQ], s_ocount[kOutQ];
    __shared__ uint64_t s_ostart[kOutQ];
    __shared__ InDesc in_desc[kSlots];
    __shared__ uint64_t s_in_end[kSlots];  // producer-private: ring end of the tile in each slot
    __shared__ uint32_t s_warp[2][kConsumerWarps];  // by tile parity: a warp may run one tile ahead

    uint32_t* err = reinterpret_cast<uint32_t*>(ws);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        for (int i = 0; i < kSlots; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], kConsumerWarps);
        }
        for (int i = 0; i < kOutQ; ++i) {
            mbar_init(&ofull[i], kConsumerWarps);  // every consumer warp has written its matches
            mbar_init(&oempty[i], 1);
        }
        s_released_out = 0;
        fence_mbar_init();
    }
    __syncthreads();

    if (warp == kProducerWarp) {
        // ------------------------------------------------------ producer --
        // Groups of kGroup consecutive tiles are handed out by a ticket
        // counter, so groups complete roughly in global order and a
        // look-back finds an inclusive prefix nearby.  Tickets are fetched
        // two groups ahead and split entries one group ahead, so neither
        // latency stalls the staging.  Lane x computes the staging parameters
        // of the group's tile x.
        uint32_t* ticket = reinterpret_cast<uint32_t*>(ws + kOffTicket);
        uint64_t head = 0, released = 0;  // virtual ring offsets (lane 0)
        uint32_t k = 0, k_rel = 0;        // tiles staged / tiles known released
        bool done = false;
        auto load_splits = [&](uint64_t grp, uint64_t& sa_, uint64_t& sb_) {
            const uint64_t idx = grp * kGroup + lane;
            sa_ = (lane <= kGroup && idx <= nTiles) ? split_a[idx] : 0;
            sb_ = (lane <= kGroup && idx <= nTiles) ? split_b[idx] : 0;
        };
        // lane 0: wait for the oldest staged tile to be released by every consumer warp
        auto wait_release = [&]() -> bool {
            const uint32_t sl = k_rel % kSlots;
            if (!mbar_wait_bounded(&empty[sl], (k_rel / kSlots) & 1, err, 2, k_rel)) return false;
            released = s_in_end[sl];
            ++k_rel;
            return true;
        };
        uint32_t tk0 = 0, tk1 = 0;
        if (lane == 0) {
            tk0 = atomicAdd(ticket, 1u);
            tk1 = atomicAdd(ticket, 1u);
        }
        uint64_t g = __shfl_sync(kFullMask, tk0, 0);
        uint64_t g_next = __shfl_sync(kFullMask, tk1, 0);
        uint64_t sp_a, sp_b;
        load_splits(g, sp_a, sp_b);
        while (!done) {
            const uint64_t t_first = g * kGroup;
            uint32_t tk2 = 0;
            if (lane == 0 && t_first < nTiles) tk2 = atomicAdd(ticket, 1u);  // two groups ahead
            uint64_t nsp_a, nsp_b;
            load_splits(g_next, nsp_a, nsp_b);  // in flight while this group is staged
            // ---- lane x: parameters of tile t_first + x ----
            uint64_t a0 = __shfl_sync(kFullMask, sp_a, lane < kGroup ? lane : 0);
            uint64_t a1 = __shfl_sync(kFullMask, sp_a, lane < kGroup ? lane + 1 : 1);
            uint64_t b0 = __shfl_sync(kFullMask, sp_b, lane < kGroup ? lane : 0);
            uint64_t b1 = __shfl_sync(kFullMask, sp_b, lane < kGroup ? lane + 1 : 1);
            const bool ok = a0 <= a1 && a1 <= nA && a1 - a0 <= kTileMax && b0 <= b1 && b1 <= nB && b1 - b0 <= kTileMax;
            const uint64_t t_mine = t_first + lane;
            if (!ok && lane < kGroup && t_mine < nTiles) record_error(err, SI_ERR_INVALID_INPUT);
            if (!ok) a0 = a1 = b0 = b1 = 0;
            // 16-byte aligned superset of [x0, x1] (x1, the successor element
            // when it exists, doubles as the merge sentinel).  Every 16-byte
            // block copied holds at least one element of the range.
            const uint64_t aEnd = a1 < nA ? a1 + 1 : a1, bEnd = b1 < nB ? b1 + 1 : b1;
            const uintptr_t a_lo = reinterpret_cast<uintptr_t>(A + a0) & ~uintptr_t(15);
            const uintptr_t b_lo = reinterpret_cast<uintptr_t>(B + b0) & ~uintptr_t(15);
            const uint32_t bytesA =
                aEnd > a0 ? static_cast<uint32_t>(((reinterpret_cast<uintptr_t>(A + aEnd) + 15) & ~uintptr_t(15)) - a_lo)
                          : 0u;
            const uint32_t bytesB =
                bEnd > b0 ? static_cast<uint32_t>(((reinterpret_cast<uintptr_t>(B + bEnd) + 15) & ~uintptr_t(15)) - b_lo)
                          : 0u;
            const uint32_t needA = bytesA / 4 + 4, needB = bytesB / 4 + 4;  // (+4: room for misalignment)
            const uint32_t misA = static_cast<uint32_t>((reinterpret_cast<uintptr_t>(A + a0) & 15u) >> 2);
            const uint32_t misB = static_cast<uint32_t>((reinterpret_cast<uintptr_t>(B + b0) & 15u) >> 2);
            const uint32_t fast = (t_mine + 1 < nTiles) && a1 < nA && b1 < nB;
            for (int x = 0; x < kGroup; ++x) {
                const uint64_t t = t_first + x;
                const uint32_t slot = k % kSlots;
                const uint64_t xa_lo = __shfl_sync(kFullMask, static_cast<uint64_t>(a_lo), x);
                const uint64_t xb_lo = __shfl_sync(kFullMask, static_cast<uint64_t>(b_lo), x);
                const uint32_t xbytesA = __shfl_sync(kFullMask, bytesA, x), xbytesB = __shfl_sync(kFullMask, bytesB, x);
                const uint32_t xneedA = __shfl_sync(kFullMask, needA, x), xneedB = __shfl_sync(kFullMask, needB, x);
                const uint32_t xmisA = __shfl_sync(kFullMask, misA, x), xmisB = __shfl_sync(kFullMask, misB, x);
                const uint32_t xna = __shfl_sync(kFullMask, static_cast<uint32_t>(a1 - a0), x);
                const uint32_t xnb = __shfl_sync(kFullMask, static_cast<uint32_t>(b1 - b0), x);
                const uint32_t xfast = __shfl_sync(kFullMask, fast, x);
                if (lane == 0) {
                    // the slot's previous tile (k - kSlots) must be released by
                    // every consumer warp before the slot is written, also for
                    // the end marker
                    bool alive = true;
                    while (alive && k_rel + kSlots <= k) alive = wait_release();
                    const bool slot_free = alive;
                    alive = alive && t < nTiles;
                    const uint32_t need = xneedA + xneedB;
                    if (alive) {
                        // A tile never wraps: if it does not fit before the ring's end it
                        // starts the next lap.  It may be placed once it overlaps no live
                        // tile: either every staged tile is released, or the live span
                        // [released, head) ends at least kRing before the tile's end.
                        const uint64_t phys = head % kRing;
                        if (phys + need > kRing) head += kRing - phys;
                        while (alive && k_rel < k && head + need - released > kRing) alive = wait_release();
                    }
                    if (!alive) {
                        if (t < nTiles) record_error(err, SI_ERR_TIMEOUT, 3, static_cast<uint32_t>(t));
                        if (slot_free) {  // else the consumers' own bounded waits end them
                            in_desc[slot].tile = kEndTile;
                            mbar_arrive(&full[slot]);
                        }
                    } else {
                        const uint32_t base = static_cast<uint32_t>(head % kRing);
                        head += need;
                        s_in_end[slot] = head;
                        InDesc& d = in_desc[slot];
                        d.tile = static_cast<uint32_t>(t);
                        d.offA = base + xmisA;
                        d.offB = base + xneedA + xmisB;
                        d.na = static_cast<int>(xna);
                        d.nb = static_cast<int>(xnb);
                        d.fast = xfast;
                        mbar_arrive_expect_tx(&full[slot], xbytesA + xbytesB);
                        if (xbytesA) bulk_g2s(in_ring + base, reinterpret_cast<const void*>(xa_lo), xbytesA, &full[slot]);
                        if (xbytesB)
                            bulk_g2s(in_ring + base + xneedA, reinterpret_cast<const void*>(xb_lo), xbytesB, &full[slot]);
                    }
                    done = !alive;
                }
                done = __shfl_sync(kFullMask, done ? 1u : 0u, 0) != 0;
                if (done) break;
                ++k;
            }
            g = g_next;
            g_next = __shfl_sync(kFullMask, tk2, 0);
            sp_a = nsp_a;
            sp_b = nsp_b;
        }
        return;
    }

    if (warp == kOutputWarp) {
        // -------------------------------------------------------- output --
        // For each tile this CTA consumed, in order: its exclusive prefix (a
        // look-back for the first tile of a group, else the running sum), its
        // inclusive prefix published, its matches copied to global memory.
        if constexpr (kOut) {
            uint64_t prefix = 0;
            for (uint32_t k = 0;; ++k) {
                const uint32_t q = k % kOutQ;
                if (!mbar_wait_bounded(&ofull[q], (k / kOutQ) & 1u, err, 4, k)) break;
                const uint32_t t = s_otile[q], count = s_ocount[q];
                const uint64_t start = s_ostart[q];
                if (t == kEndTile) break;
                if (t % kGroup == 0) prefix = t > 0 ? look_back(status, t, err) : 0;
                if (t > 0 && lane == 0) st_relaxed_u64(status + t, kFlagInc | ((prefix + count) & kValMask));
                bool overflow = false;
                for (uint32_t x = lane; x < count; x += 32) {
                    const uint64_t pos = prefix + x;
                    if (pos < out_cap) out[pos] = out_ring[(start + x) & (kOutRing - 1)];
                    else overflow = true;
                }
                if (overflow) record_error(err, SI_ERR_OUTPUT_OVERFLOW, 9, t);
                prefix += count;
                if (lane == 0 && t + 1 == nTiles) *d_count = prefix;
                __syncwarp();
                if (lane == 0) {
                    st_release_shared_u64(&s_released_out, start + count);
                    mbar_arrive(&oempty[q]);
                }
            }
        }
        return;
    }

    // ---------------------------------------------------------- consumers --
    uint64_t my_count = 0;     // count-only: this thread's matches over all its tiles
    uint64_t ohead = 0;        // element output: virtual output-ring head (same in every thread)
    uint32_t k = 0;            // tiles consumed so far
    for (;; ++k) {
        const uint32_t slot = k % kSlots;
        bool gave_up = !mbar_wait_bounded(&full[slot], (k / kSlots) & 1, err, 5, k);
        // Consumers that meet at named barriers (element output) give up
        // together: a warp leaving alone would leave the others at a barrier
        // it never reaches, which has no time limit.
        if constexpr (kOut) gave_up = named_barrier_or(kConsumerBar, kConsumers, gave_up);
        if (gave_up) break;
        const InDesc d = in_desc[slot];
        if (d.tile == kEndTile) break;
        const uint32_t* sA = in_ring + d.offA;
        const uint32_t* sB = in_ring + d.offB;
        const ThreadMatches tm = merge_inner(sA, d.na, sB, d.nb, d.fast != 0, tid);
        const uint32_t cnt = static_cast<uint32_t>(__popcll(tm.mask));

        if constexpr (!kOut) {
            my_count += cnt;
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[slot]);  // this warp is done with the tile
        } else {
            // block scan over the consumer warps
            const uint32_t incl = warp_inclusive_scan(cnt);
            if (lane == 31) s_warp[k & 1][warp] = incl;
            named_barrier(kConsumerBar, kConsumers);
            uint32_t wsum = 0, tile_count = 0;
#pragma unroll
            for (int w = 0; w < kConsumerWarps; ++w) {
                const uint32_t v = s_warp[k & 1][w];
                wsum += w < warp ? v : 0u;
                tile_count += v;
            }
            const uint32_t q = k % kOutQ;
            if (tid == 0) {
                // the tile's aggregate goes out at once, for other tiles'
                // look-backs (before the hand-off below, after which the
                // output warp overwrites it with the inclusive value)
                st_relaxed_u64(status + d.tile, (d.tile == 0 ? kFlagInc : kFlagAgg) | tile_count);
            }
            // queue entry q and ring space [ohead, ohead + tile_count) must be
            // free: the output warp has written out what they last held
            if (lane == 0) mbar_wait_bounded(&oempty[q], ((k / kOutQ) & 1u) ^ 1u, err, 7, k);
            if (lane == 0 && tile_count) {
                for (WaitBudget budget;;) {
                    if (ohead + tile_count - ld_acquire_shared_u64(&s_released_out) <= kOutRing) break;
                    if (budget.expired()) {
                        record_error(err, SI_ERR_TIMEOUT, 6, d.tile);
                        break;
                    }
                    __nanosleep(20);
                }
            }
            __syncwarp();
            uint64_t m = tm.mask;
            uint64_t pos = ohead + incl - cnt + wsum;
            while (m) {
                const int x = __ffsll(m) - 1;
                m &= m - 1;
                out_ring[pos++ & (kOutRing - 1)] = tm.src[tm.start + x];
            }
            if (tid == 0) {
                s_otile[q] = d.tile;
                s_ocount[q] = tile_count;
                s_ostart[q] = ohead;
            }
            ohead += tile_count;
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&empty[slot]);  // this warp is done with the input tile
                mbar_arrive(&ofull[q]);     // ... and has written its matches
            }
        }
    }
    if constexpr (kOut) {
        if (tid == 0) {  // end marker for the output warp (its own phase of entry q)
            const uint32_t q = k % kOutQ;
            mbar_wait_bounded(&oempty[q], ((k / kOutQ) & 1u) ^ 1u, err, 8, k);
            s_otile[q] = kEndTile;
            s_ocount[q] = 0;
            s_ostart[q] = ohead;
            for (int w = 0; w < kConsumerWarps; ++w) mbar_arrive(&ofull[q]);
        }
    } else {
        const uint64_t wsum = warp_sum_u64(my_count);
        if (lane == 0 && wsum) atomicAdd(reinterpret_cast<unsigned long long*>(d_count), wsum);
    }
}

}  // namespace

size_t ip_workspace_size(uint64_t nA, uint64_t nB, int inner) {
    return inner == kMergePath ? make_layout(nA, nB, kS).total : bm_workspace_size(nA, nB);
}

si_status ip_sisi(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB, uint64_t* d_count,
                  uint32_t* d_out, uint64_t out_cap, void* ws, size_t ws_bytes, cudaStream_t stream, int inner) {
    if (inner != kMergePath)
        return bm_sisi(dA, nA, dB, nB, d_count, d_out, out_cap, ws, ws_bytes, stream, inner == kHashProbe);
    const uint64_t S = kS;
    const Layout L = make_layout(nA, nB, S);
    if (ws_bytes < L.total) return SI_ERR_WORKSPACE_TOO_SMALL;
    if (L.nTiles > 0x7fffffffull) return SI_ERR_INVALID_ARGUMENT;
    unsigned char* w = static_cast<unsigned char*>(ws);
    uint64_t* split_a = reinterpret_cast<uint64_t*>(w + L.off_split_a);
    uint64_t* split_b = reinterpret_cast<uint64_t*>(w + L.off_split_b);
    uint64_t* status = reinterpret_cast<uint64_t*>(w + L.off_status);
    // the split kernel also clears the header, the partial counts and the
    // tiles' look-back status words
    uint32_t* samples_a = reinterpret_cast<uint32_t*>(w + L.off_samples);
    uint32_t* samples_b = samples_a + align_up(((nA + S - 1) / S) * 4, 256) / 4;
    const si_status sst = pivot_split(dA, nA, dB, nB, S, split_a, split_b, samples_a, samples_b,
                                      reinterpret_cast<uint64_t*>(w), L.off_split_a / 8, d_count, stream);
    if (sst != SI_OK) return sst;

    const uint64_t nGroups = (L.nTiles + kGroup - 1) / kGroup;
    auto launch = [&](auto kernel, uint32_t* out) -> si_status {
        const size_t smem = kTileSmem;
        SI_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
        int per_sm = 0;
        SI_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, smem));
        if (per_sm < 1) return SI_ERR_UNSUPPORTED;
        const unsigned grid =
            static_cast<unsigned>(std::min<uint64_t>(nGroups, static_cast<uint64_t>(sm_count()) * per_sm));
        uint64_t cap = out ? out_cap : 0;
        uint64_t nTiles = L.nTiles;
        void* args[] = {(void*)&dA, (void*)&nA, (void*)&dB, (void*)&nB, (void*)&split_a, (void*)&split_b,
                        (void*)&nTiles, (void*)&w, (void*)&status, (void*)&out, (void*)&cap, (void*)&d_count};
        PhaseTimer timer("sisi_tile", stream);
        SI_CUDA_TRY(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(grid), dim3(kBlock), args,
                                                smem, stream));
        return SI_OK;
    };
    const si_status st = d_out ? launch(ip_tile_kernel<true>, d_out) : launch(ip_tile_kernel<false>, nullptr);
    if (st != SI_OK) return st;
    SI_LAUNCH_CHECK("sisi_tile_kernel");
    return SI_OK;
}

}  // namespace si
