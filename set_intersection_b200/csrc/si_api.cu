// si_api.cu -- the C ABI of libsi_b200.so: argument checks, technique
// dispatch, workspace sizing, error reporting.  Declarations and the
// reference interfaces each entry point replaces are in include/si.h.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "si_device.cuh"
#include "si_internal.h"

namespace si {

namespace {
thread_local std::string g_last_error;
}

si_status cuda_fail(cudaError_t e, const char* what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return SI_ERR_CUDA;
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

namespace {

struct TimerRecord {
    const char* name = nullptr;  // the launcher's string literal
    cudaEvent_t start = nullptr, stop = nullptr;
    int device = 0;
};
std::mutex g_timer_mu;
bool g_timer_on = false;
std::vector<TimerRecord> g_timer;
// Idle events with their device: si_timer_reset returns the records' events
// here, so a timed launch records two events instead of creating them.
std::vector<std::pair<int, cudaEvent_t>> g_event_pool;

cudaEvent_t pool_take_locked(int dev) {
    for (size_t i = g_event_pool.size(); i-- > 0;) {
        if (g_event_pool[i].first != dev) continue;
        const cudaEvent_t e = g_event_pool[i].second;
        g_event_pool[i] = g_event_pool.back();
        g_event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    return cudaEventCreate(&e) == cudaSuccess ? e : nullptr;
}

}  // namespace

PhaseTimer::PhaseTimer(const char* name, cudaStream_t stream) : slot_(-1), stream_(stream) {
    std::lock_guard<std::mutex> lk(g_timer_mu);
    if (!g_timer_on) return;
    TimerRecord r;
    r.name = name;
    if (cudaGetDevice(&r.device) != cudaSuccess) return;
    r.start = pool_take_locked(r.device);
    if (!r.start) return;
    r.stop = pool_take_locked(r.device);
    if (!r.stop) {
        g_event_pool.emplace_back(r.device, r.start);
        return;
    }
    cudaEventRecord(r.start, stream);
    g_timer.push_back(r);
    slot_ = static_cast<int>(g_timer.size()) - 1;
}

PhaseTimer::~PhaseTimer() {
    if (slot_ < 0) return;
    std::lock_guard<std::mutex> lk(g_timer_mu);
    if (slot_ < static_cast<int>(g_timer.size())) cudaEventRecord(g_timer[slot_].stop, stream_);
}

namespace {

void timer_clear_locked() {
    for (auto& r : g_timer) {
        g_event_pool.emplace_back(r.device, r.start);
        g_event_pool.emplace_back(r.device, r.stop);
    }
    g_timer.clear();
}

// flag starts at 1; any descending-or-equal adjacent pair clears it.
__global__ void validate_sorted_kernel(const uint32_t* __restrict__ x, uint64_t n, uint32_t* flag) {
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    bool bad = false;
    for (uint64_t k = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x + 1; k < n; k += stride)
        bad |= __ldg(x + k - 1) >= __ldg(x + k);
    if (__any_sync(kFullMask, bad) && (threadIdx.x & 31) == 0) atomicExch(flag, 0u);
}

__global__ void set_flag_kernel(uint32_t* flag, uint32_t v) { *flag = v; }

// One thread waits, with a time limit, on an mbarrier phase that nothing
// completes: the wait must give up, record SI_ERR_TIMEOUT in the error word
// and let the kernel end.
__global__ void wait_selftest_kernel(uint32_t* err, uint64_t limit_ns) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x != 0) return;
    err[0] = err[1] = err[2] = err[3] = 0;
    mbar_init(&bar, 1);
    fence_mbar_init();
    mbar_wait_bounded(&bar, 0, err, 31, 0, limit_ns);
}

bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

}  // namespace

si_status validate_sorted(const uint32_t* d_x, uint64_t n, uint32_t* d_flag, cudaStream_t stream) {
    set_flag_kernel<<<1, 1, 0, stream>>>(d_flag, 1u);
    SI_LAUNCH_CHECK("set_flag_kernel");
    if (n > 1) {
        const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, static_cast<uint64_t>(sm_count()) * 8);
        validate_sorted_kernel<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(d_x, n, d_flag);
        SI_LAUNCH_CHECK("validate_sorted_kernel");
    }
    return SI_OK;
}

}  // namespace si

extern "C" {

const char* si_version(void) { return "set_intersection_b200 0.1.0 (sm_100a)"; }

const char* si_status_string(si_status s) {
    switch (s) {
        case SI_OK: return "ok";
        case SI_ERR_INVALID_ARGUMENT: return "invalid argument";
        case SI_ERR_WORKSPACE_TOO_SMALL: return "workspace too small";
        case SI_ERR_CUDA: return "CUDA error";
        case SI_ERR_UNSUPPORTED: return "unsupported technique for this entry point";
        case SI_ERR_TIMEOUT: return "a bounded device-side wait gave up";
        case SI_ERR_INVALID_INPUT: return "input set is not strictly increasing";
        case SI_ERR_OUTPUT_OVERFLOW: return "materialised output exceeded its capacity";
    }
    return "unknown status";
}

const char* si_last_error_string(void) { return si::g_last_error.c_str(); }

size_t si_sisi_workspace_size(uint64_t nA, uint64_t nB, si_technique t) {
    switch (t) {
        case SI_TECH_IP:
            return si::ip_workspace_size(nA, nB);
        case SI_TECH_HI:
            return si::ip_workspace_size(nA, nB, 2);
        case SI_TECH_BITMAP:
            return si::ip_workspace_size(nA, nB, 1);
        case SI_TECH_AUTO:
            return std::max(si::ip_workspace_size(nA, nB, 1), si::obs_workspace_size(nA, nB));
        case SI_TECH_OBS:
            return si::obs_workspace_size(nA, nB);
        default:
            return 0;
    }
}

si_status si_sisi(const uint32_t* dA, uint64_t nA, const uint32_t* dB, uint64_t nB, si_technique t,
                  uint64_t* d_count, uint32_t* d_out, uint64_t out_cap, void* d_workspace, size_t workspace_bytes,
                  si_stream_t stream) {
    if ((nA && !dA) || (nB && !dB) || !d_count || !d_workspace) return SI_ERR_INVALID_ARGUMENT;
    if (!si::aligned(dA, 4) || !si::aligned(dB, 4) || !si::aligned(d_count, 8) || !si::aligned(d_workspace, 16) ||
        (d_out && !si::aligned(d_out, 4)))
        return SI_ERR_INVALID_ARGUMENT;
    if (d_out && out_cap < (nA < nB ? nA : nB)) return SI_ERR_INVALID_ARGUMENT;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    switch (t) {
        case SI_TECH_IP:
            return si::ip_sisi(dA, nA, dB, nB, d_count, d_out, out_cap, d_workspace, workspace_bytes, s, 0);
        case SI_TECH_AUTO:
            // skewed pairs: search the small set in the large one (reads a
            // fraction of the large set); otherwise stream both through tiles
            if (std::min(nA, nB) * si::kSkewRatio < std::max(nA, nB))
                return si::obs_sisi(dA, nA, dB, nB, d_count, d_out, d_workspace, workspace_bytes, s);
            return si::ip_sisi(dA, nA, dB, nB, d_count, d_out, out_cap, d_workspace, workspace_bytes, s, 1);
        case SI_TECH_BITMAP:
            return si::ip_sisi(dA, nA, dB, nB, d_count, d_out, out_cap, d_workspace, workspace_bytes, s, 1);
        case SI_TECH_HI:
            return si::ip_sisi(dA, nA, dB, nB, d_count, d_out, out_cap, d_workspace, workspace_bytes, s, 2);
        case SI_TECH_OBS:
            return si::obs_sisi(dA, nA, dB, nB, d_count, d_out, d_workspace, workspace_bytes, s);
        default:
            return SI_ERR_INVALID_ARGUMENT;
    }
}

size_t si_misi_workspace_size(si_set_range A, si_set_range B, si_technique t) {
    if (t != SI_TECH_IP && t != SI_TECH_OBS && t != SI_TECH_HI && t != SI_TECH_BITMAP && t != SI_TECH_AUTO) return 0;
    if (A.end < A.start || B.end < B.start) return 0;
    return si::misi_workspace_size(A, B);
}

si_status si_misi(const uint32_t* d_elements, const uint64_t* d_offsets, si_set_range A, si_set_range B,
                  uint64_t stride, si_technique t, uint32_t* d_counts, void* d_workspace, size_t workspace_bytes,
                  si_stream_t stream) {
    if (t == SI_TECH_MM || t == SI_TECH_BITMAP_NAIVE) return SI_ERR_UNSUPPORTED;  // si_misi_dense
    if (t != SI_TECH_IP && t != SI_TECH_OBS && t != SI_TECH_HI && t != SI_TECH_BITMAP && t != SI_TECH_AUTO)
        return SI_ERR_INVALID_ARGUMENT;
    if (!d_offsets || !d_workspace || !d_counts) return SI_ERR_INVALID_ARGUMENT;
    if (A.end < A.start || B.end < B.start) return SI_ERR_INVALID_ARGUMENT;
    const bool self = A.start == B.start && A.end == B.end;
    const uint64_t nA = A.end - A.start, nB = B.end - B.start;
    if (!self && A.start < B.end && B.start < A.end) return SI_ERR_INVALID_ARGUMENT;  // overlapping ranges
    if (stride < (self ? nA : nB)) return SI_ERR_INVALID_ARGUMENT;
    if (nA + nB >= (1ull << 31)) return SI_ERR_UNSUPPORTED;
    if (!si::aligned(d_elements, 4) || !si::aligned(d_offsets, 8) || !si::aligned(d_counts, 4) ||
        !si::aligned(d_workspace, 256))
        return SI_ERR_INVALID_ARGUMENT;
    if (t == SI_TECH_AUTO) t = SI_TECH_BITMAP;
    return si::misi_tile(d_elements, d_offsets, t, A, B, stride, d_counts, d_workspace, workspace_bytes,
                         reinterpret_cast<cudaStream_t>(stream));
}

size_t si_batch_workspace_size(uint64_t npairs) { return si::batch_workspace_size(npairs); }

static si_status batch_args(const uint32_t* d_elements, const uint64_t* d_offsets, const uint32_t* d_pairs,
                            uint64_t npairs, si_technique t, uint32_t* d_counts, void* d_workspace) {
    if (t != SI_TECH_IP && t != SI_TECH_OBS && t != SI_TECH_HI && t != SI_TECH_BITMAP && t != SI_TECH_AUTO)
        return SI_ERR_INVALID_ARGUMENT;
    if (!d_offsets || !d_workspace || (npairs && (!d_pairs || !d_counts))) return SI_ERR_INVALID_ARGUMENT;
    if (npairs >= (1ull << 32)) return SI_ERR_UNSUPPORTED;
    if (!si::aligned(d_elements, 4) || !si::aligned(d_offsets, 8) || !si::aligned(d_pairs, 4) ||
        !si::aligned(d_counts, 4) || !si::aligned(d_workspace, 256))
        return SI_ERR_INVALID_ARGUMENT;
    return SI_OK;
}

si_status si_batch_count(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, const uint32_t* d_pairs,
                         uint64_t npairs, si_technique t, const uint8_t* table, uint32_t* d_counts,
                         void* d_workspace, size_t workspace_bytes, si_stream_t stream) {
    const si_status st = batch_args(d_elements, d_offsets, d_pairs, npairs, t, d_counts, d_workspace);
    if (st != SI_OK) return st;
    return si::batch_count(d_elements, d_offsets, k, d_pairs, npairs, t, table, d_counts, d_workspace,
                           workspace_bytes, reinterpret_cast<cudaStream_t>(stream));
}

si_status si_batch_tune(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, const uint32_t* d_pairs,
                        uint64_t npairs, uint32_t sample, uint32_t* d_counts, void* d_workspace,
                        size_t workspace_bytes, si_stream_t stream, uint8_t* table_out) {
    if (!table_out || sample == 0) return SI_ERR_INVALID_ARGUMENT;
    const si_status st = batch_args(d_elements, d_offsets, d_pairs, npairs, SI_TECH_AUTO, d_counts, d_workspace);
    if (st != SI_OK) return st;
    return si::batch_tune(d_elements, d_offsets, k, d_pairs, npairs, sample, d_counts, d_workspace,
                          workspace_bytes, reinterpret_cast<cudaStream_t>(stream), table_out);
}

struct si_batch_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

si_status si_batch_graph_create(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k,
                                const uint32_t* d_pairs, uint64_t npairs, si_technique t, const uint8_t* table,
                                uint32_t* d_counts, void* d_workspace, size_t workspace_bytes,
                                si_batch_graph** out) {
    if (!out) return SI_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    si_status st = batch_args(d_elements, d_offsets, d_pairs, npairs, t, d_counts, d_workspace);
    if (st != SI_OK) return st;
    if (workspace_bytes < si::batch_workspace_size(npairs)) return SI_ERR_WORKSPACE_TOO_SMALL;
    cudaStream_t cs = nullptr;
    SI_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    auto* g = new si_batch_graph;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        st = si::batch_count(d_elements, d_offsets, k, d_pairs, npairs, t, table, d_counts, d_workspace,
                             workspace_bytes, cs);
        const cudaError_t e2 = cudaStreamEndCapture(cs, &g->graph);
        if (st == SI_OK && e2 != cudaSuccess) st = si::cuda_fail(e2, "cudaStreamEndCapture");
        if (st == SI_OK) {
            e = cudaGraphInstantiate(&g->exec, g->graph, 0);
            if (e != cudaSuccess) st = si::cuda_fail(e, "cudaGraphInstantiate");
        }
    } else {
        st = si::cuda_fail(e, "cudaStreamBeginCapture");
    }
    cudaStreamDestroy(cs);
    if (st != SI_OK) {
        si_batch_graph_destroy(g);
        return st;
    }
    *out = g;
    return SI_OK;
}

si_status si_batch_graph_launch(si_batch_graph* graph, si_stream_t stream) {
    if (!graph || !graph->exec) return SI_ERR_INVALID_ARGUMENT;
    SI_CUDA_TRY(cudaGraphLaunch(graph->exec, reinterpret_cast<cudaStream_t>(stream)));
    return SI_OK;
}

void si_batch_graph_destroy(si_batch_graph* graph) {
    if (!graph) return;
    if (graph->exec) cudaGraphExecDestroy(graph->exec);
    if (graph->graph) cudaGraphDestroy(graph->graph);
    delete graph;
}

size_t si_degree_stats_workspace_size(void) { return si::degree_workspace_size(); }

si_status si_degree_stats(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, uint64_t n_elements,
                          uint64_t slots, uint32_t* d_inv, uint64_t* d_set_sum, void* d_workspace,
                          size_t workspace_bytes, si_stream_t stream) {
    if (!d_offsets || !d_workspace || (n_elements && !d_elements) || (slots && !d_inv) || (k && !d_set_sum))
        return SI_ERR_INVALID_ARGUMENT;
    if (n_elements && !slots) return SI_ERR_INVALID_ARGUMENT;
    if (!si::aligned(d_elements, 4) || !si::aligned(d_offsets, 8) || !si::aligned(d_inv, 4) ||
        !si::aligned(d_set_sum, 8) || !si::aligned(d_workspace, 256))
        return SI_ERR_INVALID_ARGUMENT;
    return si::degree_stats(d_elements, d_offsets, k, n_elements, slots, d_inv, d_set_sum, d_workspace,
                            workspace_bytes, reinterpret_cast<cudaStream_t>(stream));
}

size_t si_misi_dense_workspace_size(uint32_t k, uint32_t universe, si_technique t) {
    if (t != SI_TECH_MM && t != SI_TECH_BITMAP_NAIVE) return 0;
    if (!si::dense_supported(universe, t)) return 0;
    return si::dense_workspace_size(k, universe, t);
}

si_status si_misi_dense(const uint32_t* d_elements, const uint64_t* d_offsets, uint32_t k, uint32_t universe,
                        si_technique t, si_dense_dtype dtype, uint32_t* d_counts, void* d_workspace,
                        size_t workspace_bytes, si_stream_t stream) {
    if (t != SI_TECH_MM && t != SI_TECH_BITMAP_NAIVE) return SI_ERR_UNSUPPORTED;
    if (dtype != SI_DENSE_INT8 && dtype != SI_DENSE_FP8_E4M3) return SI_ERR_INVALID_ARGUMENT;
    if (!d_offsets || !d_workspace || (k >= 2 && !d_counts)) return SI_ERR_INVALID_ARGUMENT;
    if (!si::aligned(d_elements, 4) || !si::aligned(d_offsets, 8) || !si::aligned(d_counts, 4) ||
        !si::aligned(d_workspace, 256))
        return SI_ERR_INVALID_ARGUMENT;
    if (!si::dense_supported(universe, t)) return SI_ERR_UNSUPPORTED;
    return si::misi_dense(d_elements, d_offsets, k, universe, t, dtype == SI_DENSE_FP8_E4M3, d_counts,
                          d_workspace, workspace_bytes, reinterpret_cast<cudaStream_t>(stream));
}

si_status si_workspace_check(const void* d_workspace, si_stream_t stream) {
    if (!d_workspace) return SI_ERR_INVALID_ARGUMENT;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t code = 0;
    SI_CUDA_TRY(cudaMemcpyAsync(&code, d_workspace, sizeof(code), cudaMemcpyDeviceToHost, s));
    SI_CUDA_TRY(cudaStreamSynchronize(s));
    return static_cast<si_status>(code);
}

void si_timer_enable(int on) {
    std::lock_guard<std::mutex> lk(si::g_timer_mu);
    si::g_timer_on = on != 0;
}

void si_timer_reset(void) {
    std::lock_guard<std::mutex> lk(si::g_timer_mu);
    si::timer_clear_locked();
}

si_status si_timer_read(const char* phase, double* total_ms, uint64_t* launches) {
    if (!phase || !total_ms || !launches) return SI_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lk(si::g_timer_mu);
    double sum = 0.0;
    uint64_t n = 0;
    for (auto& r : si::g_timer) {
        if (std::strcmp(r.name, phase) != 0) continue;
        SI_CUDA_TRY(cudaEventSynchronize(r.stop));
        float ms = 0.f;
        SI_CUDA_TRY(cudaEventElapsedTime(&ms, r.start, r.stop));
        sum += ms;
        ++n;
    }
    *total_ms = sum;
    *launches = n;
    return SI_OK;
}

si_status si_workspace_diagnostic(const void* d_workspace, si_stream_t stream, uint32_t* site, uint32_t* detail) {
    if (!d_workspace || !site || !detail) return SI_ERR_INVALID_ARGUMENT;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t words[3] = {0, 0, 0};
    SI_CUDA_TRY(cudaMemcpyAsync(words, d_workspace, sizeof(words), cudaMemcpyDeviceToHost, s));
    SI_CUDA_TRY(cudaStreamSynchronize(s));
    *site = words[1];
    *detail = words[2];
    return static_cast<si_status>(words[0]);
}

si_status si_wait_selftest(void* d_workspace, uint64_t limit_ns, si_stream_t stream) {
    if (!d_workspace || !si::aligned(d_workspace, 16) || limit_ns == 0 || limit_ns > si::kWaitLimitNs)
        return SI_ERR_INVALID_ARGUMENT;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    si::wait_selftest_kernel<<<1, 32, 0, s>>>(static_cast<uint32_t*>(d_workspace), limit_ns);
    SI_LAUNCH_CHECK("wait_selftest_kernel");
    return si_workspace_check(d_workspace, stream);
}

si_status si_validate_sorted(const uint32_t* d_x, uint64_t n, uint32_t* d_flag, si_stream_t stream) {
    if ((n && !d_x) || !d_flag || !si::aligned(d_x, 4) || !si::aligned(d_flag, 4)) return SI_ERR_INVALID_ARGUMENT;
    return si::validate_sorted(d_x, n, d_flag, reinterpret_cast<cudaStream_t>(stream));
}

}  // extern "C"
