// si_misi_dense.cu -- all-pairs intersection counts of a dense collection.
//
// Two techniques for the same result, counts[tri(k, a, b)] = |S_a ∩ S_b| for
// every a < b (triangular layout of include/util.hpp:68-70):
//
//  * mm (src/matrix_multiplication.cu): the reference builds a 0/1 FP32
//    incidence matrix on the host and runs cublasSgemm per tile pair
//    (:139-184).  Here the incidence matrix M (k x U, one row per set) is
//    built on the device as 0/1 INT8 or FP8-e4m3, and C = M * M^T runs on the
//    5th-generation tensor cores: tcgen05.mma kind::i8 (s32 accumulation) or
//    kind::f8f6f4 (f32 accumulation), operands staged by TMA in 128-byte
//    swizzled K-major tiles, accumulators in tensor memory, only the tiles
//    of the upper triangle computed, only pairs a < b written.  Exact: every
//    partial sum is an integer <= U < 2^24.
//  * bitmap_naive (src/bitmap_naive.cu): every set as a bitmap, then AND +
//    popcount for every pair.  The reference gives each pair a grid-stride
//    loop and an atomic (:167-181); here it is the plain register-tiled
//    CUDA-core kernel the tensor-core path is compared against.
#include <algorithm>
#include <cstring>
#include <cuda.h>

#include "si_device.cuh"
#include "si_internal.h"

namespace si {
namespace {

// --------------------------------------------------------- tile geometry --
constexpr int kTileM = 128;        // rows of M (sets a) per tile  = TMEM lanes
constexpr int kTileN = 256;        // rows of M (sets b) per tile  = TMEM columns
constexpr int kTileK = 128;        // bytes of K per stage (one 128-byte swizzle span)
constexpr int kStages = 4;
constexpr int kMmaK = 32;          // K of one tcgen05.mma for 8-bit operands
constexpr int kBand = 8;           // row panels per rasterisation band
constexpr int kGemmThreads = 128;  // 4 warps: producer / MMA issuer / all four in the epilogue
constexpr uint32_t kStageBytesA = kTileM * kTileK;  // 16 KiB
constexpr uint32_t kStageBytesB = kTileN * kTileK;  // 32 KiB
constexpr uint32_t kStageBytes = kStageBytesA + kStageBytesB;
constexpr size_t kGemmSmem = size_t(kStages) * kStageBytes + 1024;  // + alignment slack
constexpr uint32_t kTmemCols = kTileN;  // one s32/f32 column per output column

__host__ __device__ inline uint64_t tri_index(uint64_t n, uint64_t i, uint64_t j) {
    return (n * (n - 1) / 2) - (n - i) * ((n - i) - 1) / 2 + j - i - 1;
}

// Upper-triangle tiles: tile (i, j) covers rows [128i, 128i+128) x
// [256j, 256j+256) and is needed iff it holds a pair a < b, i.e. j >= i/2.
// Order: bands of kBand row panels; in a band, column panel by column panel,
// the band's row panels inside -- so the CTAs running at the same time share
// a handful of A and B panels in L2.
__host__ __device__ inline uint32_t band_tiles(uint32_t I, uint32_t J, uint32_t b) {
    uint32_t n = 0;
    for (uint32_t i = b * kBand; i < min((b + 1) * kBand, I); ++i) n += J - i / 2;
    return n;
}

__device__ inline void tile_of(uint32_t L, uint32_t I, uint32_t J, uint32_t& ti, uint32_t& tj) {
    uint32_t b = 0;
    for (;; ++b) {
        const uint32_t n = band_tiles(I, J, b);
        if (L < n) break;
        L -= n;
    }
    const uint32_t i0 = b * kBand, i1 = min(i0 + kBand, I);
    ti = i0;
    tj = J - 1;
    for (uint32_t j = i0 / 2; j < J; ++j) {
        // row panels i of this band with i/2 <= j
        const uint32_t hi = min(i1, 2 * j + 2);
        const uint32_t cnt = hi > i0 ? hi - i0 : 0;
        if (L < cnt) {
            ti = i0 + L;
            tj = j;
            return;
        }
        L -= cnt;
    }
}

// ---------------------------------------------------------------- PTX ---
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_addr(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 128-byte swizzled, K-major operand tile: 8-row core groups of 1024 bytes
// (SBO = 1024), leading offset unused (1), descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc_sw128(const void* base) {
    const uint64_t addr = smem_addr(base);
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3fffull;             // start address
    d |= uint64_t(1) << 16;                   // leading byte offset (unused for swizzled K-major)
    d |= uint64_t(1024 >> 4) << 32;           // stride byte offset
    d |= uint64_t(1) << 46;                   // version
    d |= uint64_t(2) << 61;                   // SWIZZLE_128B
    return d;
}

// Instruction descriptor: D format, A/B formats, both K-major, N, M.
template <bool kFp8>
__host__ __device__ constexpr uint32_t instr_desc() {
    // kind::i8: D = s32 (2), A = B = unsigned 8-bit (0).  kind::f8f6f4: D = f32 (1), A = B = E4M3 (0).
    return (kFp8 ? (1u << 4) : (2u << 4)) | (uint32_t(kTileN >> 3) << 17) | (uint32_t(kTileM >> 4) << 24);
}

template <bool kFp8>
__device__ __forceinline__ void mma_issue(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    constexpr uint32_t idesc = instr_desc<kFp8>();
    if constexpr (kFp8) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
            "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
            : "memory");
    }
}

// Arrives on `bar` once every tcgen05.mma issued so far by this thread is done.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ------------------------------------------------------ incidence build --
// One CTA per row of M: the row is assembled in shared memory 32 KiB of
// columns at a time (zeros, then a `one` byte at every element of the set
// inside the chunk) and written out with 16-byte stores; rows >= k are all
// zero.  The set is read once, in order: each chunk's loop stops at the first
// element past the chunk, which is where the next chunk starts.
constexpr uint32_t kChunk = 32768;
__global__ void __launch_bounds__(256) build_incidence_kernel(const uint32_t* __restrict__ elements,
                                                              const uint64_t* __restrict__ offsets, uint32_t k,
                                                              uint8_t* __restrict__ M, uint64_t row_bytes,
                                                              uint32_t universe, uint8_t one, uint32_t* err) {
    __shared__ __align__(16) uint8_t chunk[kChunk];
    __shared__ unsigned long long s_next;
    const uint32_t row = blockIdx.x;
    uint4* c4 = reinterpret_cast<uint4*>(chunk);
    uint64_t lo = 0, e = 0;
    if (row < k) {
        lo = offsets[row];
        e = offsets[row + 1];
    }
    for (uint64_t c0 = 0; c0 < row_bytes; c0 += kChunk) {
        const uint64_t rem = row_bytes - c0;
        const uint32_t n16 = static_cast<uint32_t>((rem < kChunk ? rem : kChunk) / 16);
        for (uint32_t x = threadIdx.x; x < n16; x += blockDim.x) c4[x] = make_uint4(0, 0, 0, 0);
        if (threadIdx.x == 0) s_next = e;
        __syncthreads();
        for (uint64_t x = lo + threadIdx.x; x < e; x += blockDim.x) {
            const uint64_t v = __ldg(elements + x);
            if (v >= c0 + kChunk) {  // this thread's first element past the chunk
                atomicMin(&s_next, static_cast<unsigned long long>(x));
                break;
            }
            if (v < c0 || v > universe) { record_error(err, SI_ERR_INVALID_INPUT, 20, row); continue; }
            chunk[v - c0] = one;
        }
        __syncthreads();
        uint4* dst = reinterpret_cast<uint4*>(M + static_cast<uint64_t>(row) * row_bytes + c0);
        for (uint32_t x = threadIdx.x; x < n16; x += blockDim.x) dst[x] = c4[x];
        lo = s_next;
        __syncthreads();  // the chunk and s_next are rewritten for the next columns
    }
}

// ----------------------------------------------------- tensor-core GEMM --
template <bool kFp8>
__global__ void __launch_bounds__(kGemmThreads, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b, uint32_t k,
                   uint32_t I, uint32_t J, uint32_t num_k_stages, uint32_t* __restrict__ counts, uint32_t* err) {
    extern __shared__ uint8_t dsmem[];
    // operand stages must start on 1024-byte boundaries (swizzle atoms)
    uint8_t* stages = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(dsmem) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages], accum_full;
    __shared__ uint32_t s_tmem;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint32_t ti, tj;
    tile_of(blockIdx.x, I, J, ti, tj);

    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&accum_full, 1);
        fence_mbar_init();
    }
    if (warp == 0) {  // TMEM: 128 lanes x 256 columns of 32-bit accumulators
        tmem_alloc(&s_tmem, kTmemCols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;

    if (warp == 0 && lane == 0) {
        // ---- TMA producer ----
        for (uint32_t ks = 0; ks < num_k_stages; ++ks) {
            const uint32_t s = ks % kStages, round = ks / kStages;
            if (!mbar_wait_bounded(&empty[s], (round & 1) ^ 1, err, 21, ks)) break;
            uint8_t* sa = stages + s * kStageBytes;
            uint8_t* sb = sa + kStageBytesA;
            mbar_arrive_expect_tx(&full[s], kStageBytes);
            tma_load_2d(sa, &map_a, static_cast<int>(ks * kTileK), static_cast<int>(ti * kTileM), &full[s]);
            tma_load_2d(sb, &map_b, static_cast<int>(ks * kTileK), static_cast<int>(tj * kTileN), &full[s]);
        }
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer ----
        bool ok = true;
        for (uint32_t ks = 0; ks < num_k_stages && ok; ++ks) {
            const uint32_t s = ks % kStages, round = ks / kStages;
            ok = mbar_wait_bounded(&full[s], round & 1, err, 22, ks);
            if (!ok) break;
            tc_fence_after();
            const uint8_t* sa = stages + s * kStageBytes;
            const uint8_t* sb = sa + kStageBytesA;
            const uint64_t da = smem_desc_sw128(sa), db = smem_desc_sw128(sb);
#pragma unroll
            for (int kk = 0; kk < kTileK / kMmaK; ++kk) {
                // advance 32 bytes along K inside the swizzle span: +2 in the 16-byte address field
                mma_issue<kFp8>(tmem, da + 2 * kk, db + 2 * kk, (ks | kk) != 0);
            }
            mma_commit(&empty[s]);  // the stage is free once these MMAs have read it
        }
        mma_commit(&accum_full);
    }
    __syncwarp();

    // ---- epilogue: all four warps, warp w owns TMEM lanes (tile rows) 32w..32w+31 ----
    // warp-uniform: the TMEM loads below are .sync.aligned
    const bool done = __all_sync(kFullMask, mbar_wait_bounded(&accum_full, 0, err, 23, blockIdx.x));
    tc_fence_after();
    const uint64_t a = static_cast<uint64_t>(ti) * kTileM + warp * 32 + lane;
    const uint64_t b0 = static_cast<uint64_t>(tj) * kTileN;
    if (done) {
        // Lane l holds row a = (warp's first row) + l.  Each 32 x 32 block of
        // counts goes through a padded shared tile (the operand stages are free
        // once every MMA has completed), so that each store writes 32
        // consecutive counts of one row.
        uint32_t* blk = reinterpret_cast<uint32_t*>(stages) + warp * (32 * 33);
        const uint64_t rowbase = a < k ? tri_index(k, a, a + 1) - (a + 1) : 0;  // index of (a, b) = rowbase + b
        const uint64_t a_first = static_cast<uint64_t>(ti) * kTileM + warp * 32;
#pragma unroll 1
        for (int c = 0; c < kTileN; c += 32) {
            uint32_t v[32];
            tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c),
                      *reinterpret_cast<uint32_t(*)[16]>(v));
            tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c + 16),
                      *reinterpret_cast<uint32_t(*)[16]>(v + 16));
#pragma unroll
            for (int x = 0; x < 32; ++x)
                blk[lane * 33 + x] = kFp8 ? static_cast<uint32_t>(__uint_as_float(v[x])) : v[x];
            __syncwarp();
            const uint64_t b = b0 + c + lane;
#pragma unroll 4
            for (int r = 0; r < 32; ++r) {
                const uint64_t ar = a_first + r;
                const uint64_t base_r = __shfl_sync(kFullMask, rowbase, r);
                if (ar < k && b > ar && b < k) counts[base_r + b] = blk[r * 33 + lane];
            }
            __syncwarp();
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

// ------------------------------------------- plain AND-popcount (CUDA cores) --
// Bitmaps: one row of W 32-bit words per set (bit v of set a: word v/32, bit v%32).
__global__ void __launch_bounds__(256) build_bitmaps_kernel(const uint32_t* __restrict__ elements,
                                                            const uint64_t* __restrict__ offsets, uint32_t k,
                                                            uint32_t* __restrict__ bits, uint32_t W, uint32_t universe,
                                                            uint32_t* err) {
    extern __shared__ uint32_t row[];
    const uint32_t a = blockIdx.x;
    for (uint32_t w = threadIdx.x; w < W; w += blockDim.x) row[w] = 0u;
    __syncthreads();
    if (a < k) {
        for (uint64_t x = offsets[a] + threadIdx.x; x < offsets[a + 1]; x += blockDim.x) {
            const uint32_t v = __ldg(elements + x);
            if (v > universe) { record_error(err, SI_ERR_INVALID_INPUT, 24, a); continue; }
            atomicOr(row + (v >> 5), 1u << (v & 31));
        }
    }
    __syncthreads();
    for (uint32_t w = threadIdx.x; w < W; w += blockDim.x) bits[static_cast<uint64_t>(a) * W + w] = row[w];
}

// 128 x 128 pair tiles, 256 threads, 8 x 8 pairs per thread (rows ty + 16i,
// columns tx + 16j, so a warp's shared loads hit distinct banks or broadcast);
// K staged 16 words at a time through shared memory (double-buffered).  Only
// tiles with a < b.
constexpr int kPopTile = 128, kPopK = 16, kPopThreads = 256;
__global__ void __launch_bounds__(kPopThreads) popcount_gemm_kernel(const uint32_t* __restrict__ bits, uint32_t k,
                                                                    uint32_t W, uint32_t T,
                                                                    uint32_t* __restrict__ counts) {
    // linear upper-triangle tile index -> (ti <= tj)
    uint32_t L = blockIdx.x, ti = 0;
    while (L >= T - ti) { L -= T - ti; ++ti; }
    const uint32_t tj = ti + L;
    __shared__ uint32_t sa[2][kPopK][kPopTile + 1], sb[2][kPopK][kPopTile + 1];
    const int tid = threadIdx.x;
    const int ty = tid / 16, tx = tid % 16;  // 16 x 16 threads, 8 x 8 each
    uint32_t acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0u;
    const uint64_t rowA0 = static_cast<uint64_t>(ti) * kPopTile, rowB0 = static_cast<uint64_t>(tj) * kPopTile;
    auto load = [&](int buf, uint32_t w0) {
        for (int x = tid; x < kPopTile * kPopK; x += kPopThreads) {
            const int r = x / kPopK, c = x % kPopK;
            const uint64_t ra = rowA0 + r, rb = rowB0 + r;
            sa[buf][c][r] = (ra < k && w0 + c < W) ? __ldg(bits + ra * W + w0 + c) : 0u;
            sb[buf][c][r] = (rb < k && w0 + c < W) ? __ldg(bits + rb * W + w0 + c) : 0u;
        }
    };
    load(0, 0);
    __syncthreads();
    const uint32_t nk = (W + kPopK - 1) / kPopK;
    for (uint32_t kb = 0; kb < nk; ++kb) {
        const int buf = kb & 1;
        if (kb + 1 < nk) load(buf ^ 1, (kb + 1) * kPopK);
#pragma unroll 4
        for (int c = 0; c < kPopK; ++c) {
            uint32_t x[8], y[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) x[i] = sa[buf][c][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < 8; ++j) y[j] = sb[buf][c][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[i][j] += __popc(x[i] & y[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint64_t a = rowA0 + ty + 16 * i;
        if (a >= k) continue;
        const uint64_t rowbase = tri_index(k, a, a + 1) - (a + 1);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint64_t b = rowB0 + tx + 16 * j;
            if (b > a && b < k) counts[rowbase + b] = acc[i][j];
        }
    }
}

// ---------------------------------------------------------------- host --
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

struct DenseLayout {
    uint32_t k_pad = 0;       // rows of M (multiple of 256)
    uint64_t row_bytes = 0;   // columns of M: universe + 1 rounded up to kTileK
    uint32_t W = 0;           // bitmap words per set
    size_t off_matrix = 0, total = 0;
};
constexpr size_t kDenseHeader = 256;  // error words

DenseLayout dense_layout(uint32_t k, uint32_t universe, si_technique t) {
    DenseLayout L;
    const uint64_t U = static_cast<uint64_t>(universe) + 1;  // values 0..universe
    L.off_matrix = kDenseHeader;
    if (t == SI_TECH_BITMAP_NAIVE) {
        L.W = static_cast<uint32_t>((U + 31) / 32);
        L.total = L.off_matrix + static_cast<uint64_t>(k) * L.W * 4;
    } else {
        L.k_pad = (k + kTileN - 1) / kTileN * kTileN;
        L.row_bytes = (U + kTileK - 1) / kTileK * kTileK;
        L.total = L.off_matrix + static_cast<uint64_t>(L.k_pad) * L.row_bytes;
    }
    return L;
}

}  // namespace

size_t dense_workspace_size(uint32_t k, uint32_t universe, si_technique t) {
    return dense_layout(k, universe, t).total;
}

si_status misi_dense(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, uint32_t universe,
                     si_technique t, int fp8, uint32_t* d_counts, void* ws, size_t ws_bytes, cudaStream_t stream) {
    const DenseLayout L = dense_layout(k, universe, t);
    if (ws_bytes < L.total) return SI_ERR_WORKSPACE_TOO_SMALL;
    unsigned char* w = static_cast<unsigned char*>(ws);
    uint32_t* err = reinterpret_cast<uint32_t*>(w);
    SI_CUDA_TRY(cudaMemsetAsync(w, 0, kDenseHeader, stream));
    if (k < 2) return SI_OK;

    if (t == SI_TECH_BITMAP_NAIVE) {
        uint32_t* bits = reinterpret_cast<uint32_t*>(w + L.off_matrix);
        const size_t row_smem = static_cast<size_t>(L.W) * 4;
        if (row_smem > 200 * 1024) return SI_ERR_UNSUPPORTED;  // universe above ~6.5M values
        SI_CUDA_TRY(cudaFuncSetAttribute(build_bitmaps_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(row_smem)));
        {
            PhaseTimer timer("naive_bitmaps", stream);
            build_bitmaps_kernel<<<k, 256, row_smem, stream>>>(d_elements, d_offsets, k, bits, L.W, universe, err);
        }
        SI_LAUNCH_CHECK("build_bitmaps_kernel");
        const uint32_t T = (k + kPopTile - 1) / kPopTile;
        const uint64_t ntiles = static_cast<uint64_t>(T) * (T + 1) / 2;
        if (ntiles > 0x7fffffffull) return SI_ERR_UNSUPPORTED;
        PhaseTimer timer("naive_popcount", stream);
        popcount_gemm_kernel<<<static_cast<unsigned>(ntiles), kPopThreads, 0, stream>>>(bits, k, L.W, T, d_counts);
        SI_LAUNCH_CHECK("popcount_gemm_kernel");
        return SI_OK;
    }

    // ---- mm on tensor cores ----
    uint8_t* M = reinterpret_cast<uint8_t*>(w + L.off_matrix);
    {
        PhaseTimer timer("mm_incidence", stream);
        build_incidence_kernel<<<L.k_pad, 256, 0, stream>>>(d_elements, d_offsets, k, M, L.row_bytes, universe,
                                                         fp8 ? uint8_t(0x38) : uint8_t(1), err);  // 1.0 in e4m3 = 0x38
    }
    SI_LAUNCH_CHECK("build_incidence_kernel");

    EncodeTiledFn enc = encode_tiled();
    if (!enc) return cuda_fail(cudaErrorNotSupported, "cuTensorMapEncodeTiled unavailable");
    CUtensorMap map_a, map_b;
    const cuuint64_t gdim[2] = {L.row_bytes, L.k_pad};
    const cuuint64_t gstride[1] = {L.row_bytes};
    const cuuint32_t estride[2] = {1, 1};
    const cuuint32_t box_a[2] = {kTileK, kTileM}, box_b[2] = {kTileK, kTileN};
    const CUtensorMapDataType dt = CU_TENSOR_MAP_DATA_TYPE_UINT8;
    if (enc(&map_a, dt, 2, M, gdim, gstride, box_a, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
        enc(&map_b, dt, 2, M, gdim, gstride, box_b, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cuda_fail(cudaErrorInvalidValue, "cuTensorMapEncodeTiled");

    const uint32_t I = L.k_pad / kTileM, J = L.k_pad / kTileN;
    uint64_t ntiles = 0;
    for (uint32_t b = 0; b * kBand < I; ++b) ntiles += band_tiles(I, J, b);
    const uint32_t nks = static_cast<uint32_t>(L.row_bytes / kTileK);
    auto kern = fp8 ? tc_gemm_kernel<true> : tc_gemm_kernel<false>;
    SI_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kGemmSmem)));
    PhaseTimer timer("mm_gemm", stream);
    kern<<<static_cast<unsigned>(ntiles), kGemmThreads, kGemmSmem, stream>>>(map_a, map_b, k, I, J, nks, d_counts,
                                                                           err);
    SI_LAUNCH_CHECK("tc_gemm_kernel");
    return SI_OK;
}

}  // namespace si
