// si_host.cpp -- single pair from HOST buffers (si_sisi_host): the path of the
// reference's executables for a 2-set file (src/ip.cu:129-177: cudaMemcpy of
// the dataset, the intersection kernels, the count copied back), as one call
// that also returns the sorted elements.
//
// The pair is cut into value ranges at evenly spaced elements of the larger
// set (the smaller set is cut by a host binary search), so the intersection is
// the concatenation of the ranges' intersections.  The ranges are pipelined
// over three streams: range i's sets are copied up on one copy stream, range
// i is intersected on the caller's stream once they have landed (si_sisi into
// its own output region), its count comes back on the caller's stream, and as
// soon as the host holds that count the range's elements are copied back on a
// second copy stream to their final place in h_out.  The call therefore costs
// about the host-to-device copy of the inputs (with pinned host buffers; from
// pageable memory the copies are staged by the driver and do not overlap).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "si.h"
#include "si_internal.h"

namespace si {
namespace {

constexpr uint32_t kMaxChunks = 64;

struct Chunks {
    uint32_t n = 0;
    std::vector<uint64_t> a, b;  // n + 1 bounds each
};

Chunks split(const uint32_t* hA, uint64_t nA, const uint32_t* hB, uint64_t nB, uint32_t chunks) {
    Chunks c;
    const uint64_t n_min = std::min(nA, nB);
    uint32_t C = chunks ? chunks : ((nA + nB) >= (uint64_t(1) << 22) ? 8u : 1u);
    C = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>({C, kMaxChunks, n_min ? n_min : 1})));
    c.n = C;
    const bool a_big = nA >= nB;
    const uint32_t* big = a_big ? hA : hB;
    const uint32_t* small = a_big ? hB : hA;
    const uint64_t n_big = a_big ? nA : nB, n_small = a_big ? nB : nA;
    std::vector<uint64_t> ib(C + 1), is(C + 1);
    for (uint32_t i = 0; i <= C; ++i) ib[i] = n_big * i / C;
    is[0] = 0;
    is[C] = n_small;
    for (uint32_t i = 1; i < C; ++i) {
        const uint32_t v = big[ib[i]];
        is[i] = static_cast<uint64_t>(std::lower_bound(small, small + n_small, v) - small);
        is[i] = std::max(is[i], is[i - 1]);  // (monotone even for unsorted input)
    }
    c.a = a_big ? ib : is;
    c.b = a_big ? is : ib;
    return c;
}

struct Layout {
    size_t off_a = 0, off_b = 0, off_out = 0, off_count = 0, off_ws = 0, ws = 0, total = 0;
};

Layout layout(const Chunks& c, uint64_t nA, uint64_t nB, si_technique t) {
    Layout L;
    size_t ws = 0;
    for (uint32_t i = 0; i < c.n; ++i)
        ws = std::max(ws, si_sisi_workspace_size(c.a[i + 1] - c.a[i], c.b[i + 1] - c.b[i], t));
    size_t o = 0;
    L.off_ws = o;      o = align_up(o + ws, 256);  // first: the workspace header is where errors go
    L.ws = ws;
    L.off_a = o;       o = align_up(o + std::max<uint64_t>(nA, 1) * 4, 256);
    L.off_b = o;       o = align_up(o + std::max<uint64_t>(nB, 1) * 4, 256);
    L.off_out = o;     o = align_up(o + std::max<uint64_t>(std::min(nA, nB), 1) * 4, 256);
    L.off_count = o;   o = align_up(o + size_t(c.n) * 8, 256);
    L.total = o;
    return L;
}

struct Streams {  // the copy streams, per-range events and pinned counts of one call
    cudaStream_t up = nullptr, down = nullptr, caller = nullptr;
    std::vector<cudaEvent_t> landed, counted;
    uint64_t* hcount = nullptr;
    ~Streams() {  // every copy of the call has finished before anything is freed, also on error paths
        cudaStreamSynchronize(caller);
        if (up) cudaStreamSynchronize(up);
        if (down) cudaStreamSynchronize(down);
        for (auto e : landed) cudaEventDestroy(e);
        for (auto e : counted) cudaEventDestroy(e);
        if (up) cudaStreamDestroy(up);
        if (down) cudaStreamDestroy(down);
        if (hcount) cudaFreeHost(hcount);
    }
};

}  // namespace
}  // namespace si

extern "C" size_t si_sisi_host_workspace_size(const uint32_t* hA, uint64_t nA, const uint32_t* hB, uint64_t nB,
                                              si_technique t, uint32_t chunks) {
    if ((nA && !hA) || (nB && !hB)) return 0;
    const si::Chunks c = si::split(hA, nA, hB, nB, chunks);
    return si::layout(c, nA, nB, t).total;
}

extern "C" si_status si_sisi_host(const uint32_t* hA, uint64_t nA, const uint32_t* hB, uint64_t nB, si_technique t,
                                  uint32_t chunks, uint64_t* count, uint32_t* h_out, uint64_t out_cap,
                                  void* d_workspace, size_t workspace_bytes, si_stream_t stream) {
    if ((nA && !hA) || (nB && !hB) || !count || !d_workspace) return SI_ERR_INVALID_ARGUMENT;
    if (h_out && out_cap < std::min(nA, nB)) return SI_ERR_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(d_workspace) % 256 != 0) return SI_ERR_INVALID_ARGUMENT;
    *count = 0;
    const si::Chunks c = si::split(hA, nA, hB, nB, chunks);
    const si::Layout L = si::layout(c, nA, nB, t);
    if (workspace_bytes < L.total) return SI_ERR_WORKSPACE_TOO_SMALL;
    if (std::min(nA, nB) == 0) return SI_OK;
    unsigned char* w = static_cast<unsigned char*>(d_workspace);
    uint32_t* dA = reinterpret_cast<uint32_t*>(w + L.off_a);
    uint32_t* dB = reinterpret_cast<uint32_t*>(w + L.off_b);
    uint32_t* dOut = reinterpret_cast<uint32_t*>(w + L.off_out);
    uint64_t* dCount = reinterpret_cast<uint64_t*>(w + L.off_count);
    void* ws = w + L.off_ws;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

    si::Streams st;
    st.caller = s;
    SI_CUDA_TRY(cudaStreamCreateWithFlags(&st.up, cudaStreamNonBlocking));
    SI_CUDA_TRY(cudaStreamCreateWithFlags(&st.down, cudaStreamNonBlocking));
    st.landed.resize(c.n, nullptr);
    st.counted.resize(c.n, nullptr);
    for (uint32_t i = 0; i < c.n; ++i) {
        SI_CUDA_TRY(cudaEventCreateWithFlags(&st.landed[i], cudaEventDisableTiming));
        SI_CUDA_TRY(cudaEventCreateWithFlags(&st.counted[i], cudaEventDisableTiming));
    }
    // the copies up start after the caller's earlier work on its stream
    cudaEvent_t start = nullptr;
    SI_CUDA_TRY(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
    st.landed.push_back(start);  // destroyed with the others
    SI_CUDA_TRY(cudaEventRecord(start, s));
    SI_CUDA_TRY(cudaStreamWaitEvent(st.up, start, 0));
    for (uint32_t i = 0; i < c.n; ++i) {
        const uint64_t a0 = c.a[i], na = c.a[i + 1] - a0, b0 = c.b[i], nb = c.b[i + 1] - b0;
        if (na) SI_CUDA_TRY(cudaMemcpyAsync(dA + a0, hA + a0, na * 4, cudaMemcpyHostToDevice, st.up));
        if (nb) SI_CUDA_TRY(cudaMemcpyAsync(dB + b0, hB + b0, nb * 4, cudaMemcpyHostToDevice, st.up));
        SI_CUDA_TRY(cudaEventRecord(st.landed[i], st.up));
    }
    std::vector<uint64_t> out_at(c.n + 1, 0);  // each range's output region on the device
    for (uint32_t i = 0; i < c.n; ++i)
        out_at[i + 1] = out_at[i] + std::min(c.a[i + 1] - c.a[i], c.b[i + 1] - c.b[i]);
    // the ranges' counts land in pinned memory, so waiting for one does not
    // hold up the launches of the next
    SI_CUDA_TRY(cudaHostAlloc(reinterpret_cast<void**>(&st.hcount), size_t(c.n) * 8, cudaHostAllocDefault));
    uint64_t total = 0;
    auto copy_down = [&](uint32_t i) -> si_status {  // range i's elements, once its count is known
        SI_CUDA_TRY(cudaEventSynchronize(st.counted[i]));
        const uint64_t ci = std::min(st.hcount[i], out_at[i + 1] - out_at[i]);
        if (h_out && ci) {
            SI_CUDA_TRY(cudaStreamWaitEvent(st.down, st.counted[i], 0));
            SI_CUDA_TRY(cudaMemcpyAsync(h_out + total, dOut + out_at[i], ci * 4, cudaMemcpyDeviceToHost, st.down));
        }
        total += st.hcount[i];
        return SI_OK;
    };
    for (uint32_t i = 0; i < c.n; ++i) {
        const uint64_t a0 = c.a[i], na = c.a[i + 1] - a0, b0 = c.b[i], nb = c.b[i + 1] - b0;
        SI_CUDA_TRY(cudaStreamWaitEvent(s, st.landed[i], 0));
        const uint64_t cap = out_at[i + 1] - out_at[i];
        const si_status r = si_sisi(dA + a0, na, dB + b0, nb, t, dCount + i, h_out && cap ? dOut + out_at[i] : nullptr,
                                    cap, ws, L.ws, stream);
        if (r != SI_OK) return r;  // (the destructor waits for the copies in flight)
        SI_CUDA_TRY(cudaMemcpyAsync(st.hcount + i, dCount + i, 8, cudaMemcpyDeviceToHost, s));
        SI_CUDA_TRY(cudaEventRecord(st.counted[i], s));
        if (i > 0) {
            const si_status d = copy_down(i - 1);
            if (d != SI_OK) return d;
        }
    }
    const si_status d = copy_down(c.n - 1);
    if (d != SI_OK) return d;
    SI_CUDA_TRY(cudaStreamSynchronize(st.down));
    *count = total;
    return si_workspace_check(ws, stream);
}
