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
// its own output region), its count and error word come back on the caller's
// stream, and as soon as the host holds that count the range's elements are
// copied back on a second copy stream to their final place in h_out.  The call
// therefore costs about the host-to-device copy of the inputs.  Pinned input
// buffers are copied by the DMA engine directly; a pageable input is staged
// through the context's pinned buffers: host threads copy 16 MiB pieces into
// them while the DMA engine moves the previous pieces up (the driver's own
// staging of pageable copies runs one piece at a time).
//
// The copy streams, the per-range events, the pinned words the counts and
// error words land in and the staging buffers belong to a si_host_ctx, created
// once (si_host_ctx_create) and reused by every si_sisi_host_ctx call (one
// call at a time per context); si_sisi_host creates and destroys one per call.
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "si.h"
#include "si_internal.h"

namespace si {
namespace {

// Host threads that copy one buffer together (fork-join): the caller takes
// the first slice, the workers the others.
class CopyPool {
public:
    explicit CopyPool(unsigned threads) {
        workers_.reserve(threads);
        for (unsigned i = 1; i < threads; ++i) {
            try {
                workers_.emplace_back([this, i] { loop(i); });
            } catch (...) {  // fewer threads than asked for: the caller's share grows
                break;
            }
        }
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
            ++gen_;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    void copy(void* dst, const void* src, size_t n) {
        {
            std::lock_guard<std::mutex> lk(m_);
            dst_ = static_cast<unsigned char*>(dst);
            src_ = static_cast<const unsigned char*>(src);
            n_ = n;
            pending_ = static_cast<unsigned>(workers_.size());
            ++gen_;
        }
        cv_.notify_all();
        part(0);
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [this] { return pending_ == 0; });
    }

private:
    void part(unsigned i) const {
        const size_t parts = workers_.size() + 1;
        const size_t step = ((n_ + parts - 1) / parts + 63) & ~size_t(63);
        const size_t lo = std::min(n_, step * i), hi = std::min(n_, lo + step);
        if (hi > lo) std::memcpy(dst_ + lo, src_ + lo, hi - lo);
    }
    void loop(unsigned i) {
        uint64_t seen = 0;
        for (;;) {
            std::unique_lock<std::mutex> lk(m_);
            cv_.wait(lk, [&] { return gen_ != seen; });
            seen = gen_;
            if (stop_) return;
            lk.unlock();
            part(i);
            lk.lock();
            if (--pending_ == 0) done_.notify_one();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    unsigned char* dst_ = nullptr;
    const unsigned char* src_ = nullptr;
    size_t n_ = 0;
    unsigned pending_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

}  // namespace
}  // namespace si

struct si_host_ctx {
    static constexpr uint32_t kMaxChunks = 64;
    static constexpr uint32_t kStages = 4;                // staging buffers for pageable inputs
    static constexpr size_t kStageBytes = size_t(16) << 20;
    int device = -1;
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t start = nullptr;
    cudaEvent_t landed[kMaxChunks] = {}, counted[kMaxChunks] = {};
    uint64_t* hcount = nullptr;  // pinned [kMaxChunks]
    uint32_t* herr = nullptr;    // pinned [kMaxChunks][4]: each range's workspace error header
    // made at the first call with a pageable input
    unsigned char* stage[kStages] = {};
    cudaEvent_t stage_free[kStages] = {};  // the last copy up from the buffer has finished
    uint32_t next_stage = 0;
    si::CopyPool* pool = nullptr;
};

namespace si {
namespace {

constexpr uint32_t kMaxChunks = si_host_ctx::kMaxChunks;

struct Chunks {
    uint32_t n = 0;
    std::vector<uint64_t> a, b;   // n + 1 bounds each
    bool descent_at_cut = false;  // a set descends across a range boundary
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
        // no range's kernels see the two elements either side of a cut
        if (ib[i] > 0 && big[ib[i] - 1] >= big[ib[i]]) c.descent_at_cut = true;
        if (is[i] > 0 && is[i] < n_small && small[is[i] - 1] >= small[is[i]]) c.descent_at_cut = true;
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

// Host-side checks of a call, made before any CUDA call.  SI_OK with `done`
// set means the result is final without a launch (an empty set).
si_status host_args(const uint32_t* hA, uint64_t nA, const uint32_t* hB, uint64_t nB, si_technique t,
                    uint32_t chunks, uint64_t* count, uint32_t* h_out, uint64_t out_cap, void* d_workspace,
                    size_t workspace_bytes, Chunks& c, Layout& L, bool& done) {
    done = false;
    if ((nA && !hA) || (nB && !hB) || !count || !d_workspace) return SI_ERR_INVALID_ARGUMENT;
    if (h_out && out_cap < std::min(nA, nB)) return SI_ERR_INVALID_ARGUMENT;
    if (reinterpret_cast<uintptr_t>(d_workspace) % 256 != 0) return SI_ERR_INVALID_ARGUMENT;
    *count = 0;
    c = split(hA, nA, hB, nB, chunks);
    L = layout(c, nA, nB, t);
    if (workspace_bytes < L.total) return SI_ERR_WORKSPACE_TOO_SMALL;
    if (std::min(nA, nB) == 0) {
        done = true;
        return SI_OK;
    }
    if (c.descent_at_cut) return SI_ERR_INVALID_INPUT;
    return SI_OK;
}

// Every copy of a call has finished before the call returns, on error paths
// too (the caller may free or reuse its host buffers at once).
struct Drain {
    si_host_ctx* ctx;
    cudaStream_t caller;
    ~Drain() {
        cudaStreamSynchronize(caller);
        cudaStreamSynchronize(ctx->up);
        cudaStreamSynchronize(ctx->down);
    }
};

// True for memory the DMA engine can read directly (cudaHostAlloc'd or
// registered); pageable memory is staged.
bool host_pinned(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

si_status ensure_staging(si_host_ctx* ctx) {
    if (ctx->pool) return SI_OK;
    for (uint32_t k = 0; k < si_host_ctx::kStages; ++k) {
        SI_CUDA_TRY(cudaHostAlloc(reinterpret_cast<void**>(&ctx->stage[k]), si_host_ctx::kStageBytes,
                                  cudaHostAllocDefault));
        SI_CUDA_TRY(cudaEventCreateWithFlags(&ctx->stage_free[k], cudaEventDisableTiming));
    }
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    ctx->pool = new (std::nothrow) CopyPool(std::min(8u, hw));
    return ctx->pool ? SI_OK : SI_ERR_UNSUPPORTED;
}

// bytes from host src to device dst on the context's up stream: directly from
// pinned memory, else through the staging buffers (a buffer is refilled once
// its previous copy up has finished; the host copy of one piece overlaps the
// DMA of the pieces before it).
si_status upload(si_host_ctx* ctx, void* dst, const void* src, size_t bytes, bool pinned) {
    if (bytes == 0) return SI_OK;
    if (pinned) {
        SI_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->up));
        return SI_OK;
    }
    for (size_t off = 0; off < bytes; off += si_host_ctx::kStageBytes) {
        const size_t n = std::min(si_host_ctx::kStageBytes, bytes - off);
        const uint32_t k = ctx->next_stage;
        ctx->next_stage = (k + 1) % si_host_ctx::kStages;
        SI_CUDA_TRY(cudaEventSynchronize(ctx->stage_free[k]));
        ctx->pool->copy(ctx->stage[k], static_cast<const unsigned char*>(src) + off, n);
        SI_CUDA_TRY(cudaMemcpyAsync(static_cast<unsigned char*>(dst) + off, ctx->stage[k], n, cudaMemcpyHostToDevice,
                                    ctx->up));
        SI_CUDA_TRY(cudaEventRecord(ctx->stage_free[k], ctx->up));
    }
    return SI_OK;
}

}  // namespace
}  // namespace si

extern "C" si_status si_host_ctx_create(si_host_ctx** out) {
    if (!out) return SI_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto* c = new si_host_ctx;
    auto fail = [&](cudaError_t e, const char* what) {
        si_host_ctx_destroy(c);
        return si::cuda_fail(e, what);
    };
    cudaError_t e = cudaGetDevice(&c->device);
    if (e != cudaSuccess) return fail(e, "cudaGetDevice");
    if ((e = cudaStreamCreateWithFlags(&c->up, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    if ((e = cudaStreamCreateWithFlags(&c->down, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    if ((e = cudaEventCreateWithFlags(&c->start, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    for (uint32_t i = 0; i < si::kMaxChunks; ++i) {
        if ((e = cudaEventCreateWithFlags(&c->landed[i], cudaEventDisableTiming)) != cudaSuccess)
            return fail(e, "event");
        if ((e = cudaEventCreateWithFlags(&c->counted[i], cudaEventDisableTiming)) != cudaSuccess)
            return fail(e, "event");
    }
    if ((e = cudaHostAlloc(reinterpret_cast<void**>(&c->hcount), si::kMaxChunks * 8, cudaHostAllocDefault)) !=
        cudaSuccess)
        return fail(e, "cudaHostAlloc");
    if ((e = cudaHostAlloc(reinterpret_cast<void**>(&c->herr), si::kMaxChunks * 16, cudaHostAllocDefault)) !=
        cudaSuccess)
        return fail(e, "cudaHostAlloc");
    *out = c;
    return SI_OK;
}

extern "C" void si_host_ctx_destroy(si_host_ctx* c) {
    if (!c) return;
    if (c->up) cudaStreamSynchronize(c->up);
    if (c->down) cudaStreamSynchronize(c->down);
    for (uint32_t i = 0; i < si::kMaxChunks; ++i) {
        if (c->landed[i]) cudaEventDestroy(c->landed[i]);
        if (c->counted[i]) cudaEventDestroy(c->counted[i]);
    }
    if (c->start) cudaEventDestroy(c->start);
    if (c->up) cudaStreamDestroy(c->up);
    if (c->down) cudaStreamDestroy(c->down);
    if (c->hcount) cudaFreeHost(c->hcount);
    if (c->herr) cudaFreeHost(c->herr);
    for (uint32_t k = 0; k < si_host_ctx::kStages; ++k) {
        if (c->stage_free[k]) cudaEventDestroy(c->stage_free[k]);
        if (c->stage[k]) cudaFreeHost(c->stage[k]);
    }
    delete c->pool;
    delete c;
}

extern "C" size_t si_sisi_host_workspace_size(const uint32_t* hA, uint64_t nA, const uint32_t* hB, uint64_t nB,
                                              si_technique t, uint32_t chunks) {
    if ((nA && !hA) || (nB && !hB)) return 0;
    const si::Chunks c = si::split(hA, nA, hB, nB, chunks);
    return si::layout(c, nA, nB, t).total;
}

extern "C" si_status si_sisi_host_ctx(si_host_ctx* ctx, const uint32_t* hA, uint64_t nA, const uint32_t* hB,
                                      uint64_t nB, si_technique t, uint32_t chunks, uint64_t* count, uint32_t* h_out,
                                      uint64_t out_cap, void* d_workspace, size_t workspace_bytes,
                                      si_stream_t stream) {
    if (!ctx) return SI_ERR_INVALID_ARGUMENT;
    si::Chunks c;
    si::Layout L;
    bool done = false;
    const si_status arg = si::host_args(hA, nA, hB, nB, t, chunks, count, h_out, out_cap, d_workspace,
                                        workspace_bytes, c, L, done);
    if (arg != SI_OK || done) return arg;
    int dev = -1;
    SI_CUDA_TRY(cudaGetDevice(&dev));
    if (dev != ctx->device) return SI_ERR_INVALID_ARGUMENT;  // the context's streams live on another device
    unsigned char* w = static_cast<unsigned char*>(d_workspace);
    uint32_t* dA = reinterpret_cast<uint32_t*>(w + L.off_a);
    uint32_t* dB = reinterpret_cast<uint32_t*>(w + L.off_b);
    uint32_t* dOut = reinterpret_cast<uint32_t*>(w + L.off_out);
    uint64_t* dCount = reinterpret_cast<uint64_t*>(w + L.off_count);
    void* ws = w + L.off_ws;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

    const bool pinned_a = si::host_pinned(hA), pinned_b = si::host_pinned(hB);
    const bool staged = !pinned_a || !pinned_b;
    if (staged) {
        const si_status st = si::ensure_staging(ctx);
        if (st != SI_OK) return st;
    }
    si::Drain drain{ctx, s};
    // the copies up start after the caller's earlier work on its stream
    SI_CUDA_TRY(cudaEventRecord(ctx->start, s));
    SI_CUDA_TRY(cudaStreamWaitEvent(ctx->up, ctx->start, 0));
    auto upload_range = [&](uint32_t i) -> si_status {
        const uint64_t a0 = c.a[i], na = c.a[i + 1] - a0, b0 = c.b[i], nb = c.b[i + 1] - b0;
        si_status st = si::upload(ctx, dA + a0, hA + a0, na * 4, pinned_a);
        if (st == SI_OK) st = si::upload(ctx, dB + b0, hB + b0, nb * 4, pinned_b);
        if (st != SI_OK) return st;
        SI_CUDA_TRY(cudaEventRecord(ctx->landed[i], ctx->up));
        return SI_OK;
    };
    // pinned inputs: every copy up is queued at once; staged ones are copied
    // range by range, each range's kernels queued as soon as its copies are
    if (!staged) {
        for (uint32_t i = 0; i < c.n; ++i) {
            const si_status st = upload_range(i);
            if (st != SI_OK) return st;
        }
    }
    std::vector<uint64_t> out_at(c.n + 1, 0);  // each range's output region on the device
    for (uint32_t i = 0; i < c.n; ++i)
        out_at[i + 1] = out_at[i] + std::min(c.a[i + 1] - c.a[i], c.b[i + 1] - c.b[i]);
    uint64_t total = 0;
    si_status first_error = SI_OK;
    // range i's elements, once its count is known; and its error word: every
    // range reuses the one workspace, whose header each range's kernels clear
    auto copy_down = [&](uint32_t i) -> si_status {
        SI_CUDA_TRY(cudaEventSynchronize(ctx->counted[i]));
        if (first_error == SI_OK && ctx->herr[4 * i] != 0) first_error = static_cast<si_status>(ctx->herr[4 * i]);
        const uint64_t ci = std::min(ctx->hcount[i], out_at[i + 1] - out_at[i]);
        if (h_out && ci) {
            SI_CUDA_TRY(cudaStreamWaitEvent(ctx->down, ctx->counted[i], 0));
            SI_CUDA_TRY(cudaMemcpyAsync(h_out + total, dOut + out_at[i], ci * 4, cudaMemcpyDeviceToHost, ctx->down));
        }
        total += ctx->hcount[i];
        return SI_OK;
    };
    for (uint32_t i = 0; i < c.n; ++i) {
        if (staged) {
            const si_status st = upload_range(i);
            if (st != SI_OK) return st;
        }
        const uint64_t a0 = c.a[i], na = c.a[i + 1] - a0, b0 = c.b[i], nb = c.b[i + 1] - b0;
        SI_CUDA_TRY(cudaStreamWaitEvent(s, ctx->landed[i], 0));
        const uint64_t cap = out_at[i + 1] - out_at[i];
        const si_status r = si_sisi(dA + a0, na, dB + b0, nb, t, dCount + i, h_out && cap ? dOut + out_at[i] : nullptr,
                                    cap, ws, L.ws, stream);
        if (r != SI_OK) return r;  // (drain waits for the copies in flight)
        SI_CUDA_TRY(cudaMemcpyAsync(ctx->hcount + i, dCount + i, 8, cudaMemcpyDeviceToHost, s));
        SI_CUDA_TRY(cudaMemcpyAsync(ctx->herr + 4 * i, ws, 16, cudaMemcpyDeviceToHost, s));
        SI_CUDA_TRY(cudaEventRecord(ctx->counted[i], s));
        if (i > 0) {
            const si_status d = copy_down(i - 1);
            if (d != SI_OK) return d;
        }
    }
    const si_status d = copy_down(c.n - 1);
    if (d != SI_OK) return d;
    SI_CUDA_TRY(cudaStreamSynchronize(ctx->down));
    *count = total;
    return first_error;
}

extern "C" si_status si_sisi_host(const uint32_t* hA, uint64_t nA, const uint32_t* hB, uint64_t nB, si_technique t,
                                  uint32_t chunks, uint64_t* count, uint32_t* h_out, uint64_t out_cap,
                                  void* d_workspace, size_t workspace_bytes, si_stream_t stream) {
    {  // argument errors and empty sets need no context
        si::Chunks c;
        si::Layout L;
        bool done = false;
        const si_status arg = si::host_args(hA, nA, hB, nB, t, chunks, count, h_out, out_cap, d_workspace,
                                            workspace_bytes, c, L, done);
        if (arg != SI_OK || done) return arg;
    }
    si_host_ctx* ctx = nullptr;
    si_status st = si_host_ctx_create(&ctx);
    if (st != SI_OK) return st;
    st = si_sisi_host_ctx(ctx, hA, nA, hB, nB, t, chunks, count, h_out, out_cap, d_workspace, workspace_bytes, stream);
    si_host_ctx_destroy(ctx);
    return st;
}
