// si_degree.cu -- the dataset statistics of the reference's degree_cdf tool
// (src/degree_cdf.cpp:19-62), computed on the device: the inverted-list
// length of every value (how many sets hold it) and, per set, the sum of its
// values' inverted-list lengths.  Sorting the two lists by their keys and the
// running sums (the CDF files) stay with the caller, whose std::sort fixes the
// order among equal keys exactly as the reference's does.
//
//  degree_inv_kernel  one thread per element: red.add of 1 into the value's
//      slot (the slots live in L2 for universes up to tens of millions).
//  degree_sum_kernel  one warp per set: gathers its elements' slots with
//      coalesced element loads and reduces them in 64 bits.
#include <algorithm>

#include "si_device.cuh"
#include "si_internal.h"

namespace si {
namespace {

constexpr size_t kDegreeHeader = 256;  // [0..16) error words

__global__ void degree_inv_kernel(const uint32_t* __restrict__ el, uint64_t n, uint64_t slots,
                                  uint32_t* __restrict__ inv, uint32_t* err) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t v = __ldg(el + i);
        if (v < slots)
            atomicAdd(inv + v, 1u);
        else
            record_error(err, SI_ERR_INVALID_INPUT, 60, static_cast<uint32_t>(i));
    }
}

__global__ void degree_sum_kernel(const uint32_t* __restrict__ el, const uint64_t* __restrict__ off, uint32_t k,
                                  uint64_t slots, const uint32_t* __restrict__ inv, uint64_t* __restrict__ set_sum) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x / 32);
    for (uint64_t s = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / 32; s < k; s += warps) {
        const uint64_t e0 = off[s], e1 = off[s + 1];
        uint64_t sum = 0;
        for (uint64_t e = e0 + lane; e < e1; e += 32) {
            const uint32_t v = __ldg(el + e);
            sum += v < slots ? __ldcg(inv + v) : 0u;  // out-of-range values are recorded by the first kernel
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) sum += __shfl_xor_sync(kFullMask, sum, d);
        if (lane == 0) set_sum[s] = sum;
    }
}

}  // namespace

size_t degree_workspace_size() { return kDegreeHeader; }

si_status degree_stats(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, uint64_t n_elements,
                       uint64_t slots, uint32_t* d_inv, uint64_t* d_set_sum, void* ws, size_t ws_bytes,
                       cudaStream_t stream) {
    if (ws_bytes < kDegreeHeader) return SI_ERR_WORKSPACE_TOO_SMALL;
    uint32_t* err = static_cast<uint32_t*>(ws);
    SI_CUDA_TRY(cudaMemsetAsync(ws, 0, kDegreeHeader, stream));
    if (slots) SI_CUDA_TRY(cudaMemsetAsync(d_inv, 0, slots * 4, stream));
    const unsigned blocks = static_cast<unsigned>(sm_count()) * 8;
    PhaseTimer timer("degree_stats", stream);
    if (n_elements) {
        degree_inv_kernel<<<blocks, 256, 0, stream>>>(d_elements, n_elements, slots, d_inv, err);
        SI_LAUNCH_CHECK("degree_inv_kernel");
    }
    if (k) {
        degree_sum_kernel<<<blocks, 256, 0, stream>>>(d_elements, d_offsets, k, slots, d_inv, d_set_sum);
        SI_LAUNCH_CHECK("degree_sum_kernel");
    }
    return SI_OK;
}

}  // namespace si
