// si_internal.h -- host-side interfaces between the C-ABI layer (si_api.cu)
// and the per-technique launchers.  Not installed; C++ only.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "si.h"

namespace si {

// Records a CUDA error text for si_last_error_string and returns SI_ERR_CUDA.
si_status cuda_fail(cudaError_t e, const char* what);

#define SI_CUDA_TRY(expr)                                                 \
    do {                                                                  \
        cudaError_t si_e_ = (expr);                                       \
        if (si_e_ != cudaSuccess) return ::si::cuda_fail(si_e_, #expr);   \
    } while (0)

#define SI_LAUNCH_CHECK(what)                                             \
    do {                                                                  \
        cudaError_t si_e_ = cudaGetLastError();                           \
        if (si_e_ != cudaSuccess) return ::si::cuda_fail(si_e_, what);    \
    } while (0)

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Number of SMs of the current device (cached per device).
int sm_count();

// Launches `kernel` with programmatic stream serialization: it may start while
// the previous kernel on the stream finishes, and must execute
// griddepcontrol.wait before it reads that kernel's results (or writes what
// that kernel still reads).
template <class Kernel, class... Args>
si_status launch_dependent(Kernel kernel, dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    SI_CUDA_TRY(cudaLaunchKernelEx(&cfg, kernel, args...));
    return SI_OK;
}

// Named phase timing on the launching stream (the engine's counterpart of the
// reference's DeviceTimer, include/device_timer.cuh:20-78).  When enabled via
// si_timer_enable, PhaseTimer records a cudaEvent pair around a launch.
class PhaseTimer {
public:
    PhaseTimer(const char* name, cudaStream_t stream);
    ~PhaseTimer();
    PhaseTimer(const PhaseTimer&) = delete;
    PhaseTimer& operator=(const PhaseTimer&) = delete;
private:
    int slot_;
    cudaStream_t stream_;
};

// ---- single-pair tile pipeline (si_sisi_ip.cu, si_sisi_bitmap.cu) ----
// inner: 0 = merge path (technique ip), 1 = the bitmap engine (technique
// bitmap: per-warp bitmap build + probe, si_sisi_bitmap.cu), 2 = hash probe
// (technique hi).  The bitmap engine's workspace is larger (its scratch array).
size_t ip_workspace_size(uint64_t nA, uint64_t nB, int inner = 0);
// Value-pivot split of (A, B) at every S-th element of each set into
// split_a/split_b[nA/S + nB/S + 2] (rounded up), through the sample arrays
// samples_a/samples_b (pivot_samples_bytes in all, two 256-byte aligned
// parts); also clears zero[0, nzero) and *d_count.  Lets the next kernel on
// the stream start early (programmatic dependent launch); that kernel must
// execute griddepcontrol.wait before it reads any of these.
si_status pivot_split(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB, uint64_t S,
                      uint64_t* split_a, uint64_t* split_b, uint32_t* samples_a, uint32_t* samples_b,
                      uint64_t* zero, uint64_t nzero, uint64_t* d_count, cudaStream_t stream);
size_t pivot_samples_bytes(uint64_t nA, uint64_t nB, uint64_t S);
// The stream engine of si_sisi_bitmap.cu: window bitmaps (technique bitmap)
// or, with hash set, window hash tables (technique hi) on the same ranges.
size_t bm_workspace_size(uint64_t nA, uint64_t nB);
si_status bm_sisi(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB, uint64_t* d_count,
                  uint32_t* d_out, uint64_t out_cap, void* ws, size_t ws_bytes, cudaStream_t stream,
                  bool hash = false);
// SI_TECH_AUTO searches the smaller set in the larger (obs) when the sizes
// differ by more than this factor.
constexpr uint64_t kSkewRatio = 64;
size_t obs_workspace_size(uint64_t nA, uint64_t nB);
si_status obs_sisi(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB, uint64_t* d_count,
                   uint32_t* d_out, void* ws, size_t ws_bytes, cudaStream_t stream);
si_status ip_sisi(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB, uint64_t* d_count,
                  uint32_t* d_out, uint64_t out_cap, void* ws, size_t ws_bytes, cudaStream_t stream, int inner = 0);

// ---- all pairs of a dense collection (si_misi_dense.cu) ----
// t: SI_TECH_MM (tensor cores; fp8 selects FP8-e4m3 operands instead of INT8)
// or SI_TECH_BITMAP_NAIVE (plain AND-popcount on CUDA cores).
size_t misi_workspace_size(si_set_range A, si_set_range B);
si_status misi_tile(const uint32_t* d_elements, const uint64_t* d_offsets, si_technique t, si_set_range A,
                    si_set_range B, uint64_t stride, uint32_t* d_counts, void* ws, size_t ws_bytes,
                    cudaStream_t stream);
size_t batch_workspace_size(uint64_t npairs);
si_status batch_count(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, const uint32_t* d_pairs,
                      uint64_t npairs, si_technique t, const uint8_t* table, uint32_t* d_counts, void* ws,
                      size_t ws_bytes, cudaStream_t stream);
si_status batch_tune(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, const uint32_t* d_pairs,
                     uint64_t npairs, uint32_t sample, uint32_t* d_counts, void* ws, size_t ws_bytes,
                     cudaStream_t stream, uint8_t* table_out);
size_t degree_workspace_size();
si_status degree_stats(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, uint64_t n_elements,
                       uint64_t slots, uint32_t* d_inv, uint64_t* d_set_sum, void* ws, size_t ws_bytes,
                       cudaStream_t stream);
// The dense path's range: MM needs every count exact in f32 (universe < 2^24);
// BITMAP_NAIVE builds one set's bitmap in shared memory (<= 200 KiB).
inline bool dense_supported(uint32_t universe, si_technique t) {
    if (t == SI_TECH_MM) return universe < (1u << 24);
    return (static_cast<uint64_t>(universe) + 32) / 32 * 4 <= 200 * 1024;
}
size_t dense_workspace_size(uint32_t k, uint32_t universe, si_technique t);
si_status misi_dense(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, uint32_t universe,
                     si_technique t, int fp8, uint32_t* d_counts, void* ws, size_t ws_bytes, cudaStream_t stream);

// ---- sortedness check (si_api.cu) ----
si_status validate_sorted(const uint32_t* d_x, uint64_t n, uint32_t* d_flag, cudaStream_t stream);

}  // namespace si
