// si_sisi_noalloc.cu -- the single-pair intersect-path call for callers that
// cannot allocate device memory.
//
// Some hosts hand this library raw device pointers but have no way to obtain
// scratch memory for it: FFI callers (cgo, JNI, ctypes) that only receive
// buffers owned by another runtime and have no CUDA allocator binding of their
// own, engines whose memory manager has already reserved the whole HBM budget,
// and latency-critical paths where cudaMalloc/cudaFree would synchronise the
// device behind other streams' backs.  si_sisi_noalloc runs exactly the
// kernels of si_sisi (technique ip) but takes its scratch from a fixed array
// in device memory that belongs to this library instead of from the caller.
//
// The array lives in every GPU that loads the library, until the process
// exits.  Host code cannot use the array's name as a device address (in host
// code it names a host-side stand-in), so the first call on each device looks
// up the real address with cudaGetSymbolAddress while that device is current
// and caches it; that first call should therefore happen before any stream
// capture.  Every call shares the one array and finds the previous call's
// contents in it: the kernels clear the parts that must start at zero on each
// call, and calls whose kernels overlap on the GPU (different streams, no
// ordering between them) race on the array and must not be issued.
#include <mutex>

#include "si_device.cuh"
#include "si_internal.h"

namespace si {
namespace {

// 4 MiB: the intersect-path scratch for any pair with |A| + |B| <= 2^29.
constexpr size_t kNoAllocScratchBytes = size_t(4) << 20;
constexpr uint64_t kNoAllocMaxElements = uint64_t(1) << 29;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (looked up once
// per device, with that device current).
si_status scratch_address(void** out) {
    int dev = 0;
    SI_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return SI_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (g_scratch_addr[dev] == nullptr) {
        void* p = nullptr;
        SI_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return SI_OK;
}

bool aligned_to(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

}  // namespace
}  // namespace si

extern "C" si_status si_sisi_noalloc(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB,
                                     uint64_t* d_count, uint32_t* d_out, uint64_t out_cap, si_stream_t stream) {
    // Host-side checks first: nothing below touches the GPU until they pass.
    if ((nA && !dA) || (nB && !dB) || !d_count) return SI_ERR_INVALID_ARGUMENT;
    if (!si::aligned_to(dA, 4) || !si::aligned_to(dB, 4) || !si::aligned_to(d_count, 8) ||
        (d_out && !si::aligned_to(d_out, 4)))
        return SI_ERR_INVALID_ARGUMENT;
    if (d_out && out_cap < (nA < nB ? nA : nB)) return SI_ERR_INVALID_ARGUMENT;
    if (nA > si::kNoAllocMaxElements || nB > si::kNoAllocMaxElements || nA + nB > si::kNoAllocMaxElements ||
        si::ip_workspace_size(nA, nB) > si::kNoAllocScratchBytes)
        return SI_ERR_WORKSPACE_TOO_SMALL;
    void* scratch = nullptr;
    si_status st = si::scratch_address(&scratch);
    if (st != SI_OK) return st;
    return si::ip_sisi(dA, nA, dB, nB, d_count, d_out, out_cap, scratch, si::kNoAllocScratchBytes,
                       reinterpret_cast<cudaStream_t>(stream));
}

extern "C" si_status si_sisi_noalloc_check(si_stream_t stream) {
    // the error words of the library's scratch array, read into host memory:
    // copies from a symbol allocate nothing
    uint32_t words[4] = {0, 0, 0, 0};
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    SI_CUDA_TRY(cudaMemcpyFromSymbolAsync(words, si::g_noalloc_scratch, sizeof(words), 0, cudaMemcpyDeviceToHost, s));
    SI_CUDA_TRY(cudaStreamSynchronize(s));
    return static_cast<si_status>(words[0]);
}
