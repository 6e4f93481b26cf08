// si_device.cuh -- device-side building blocks shared by the sm_100a kernels:
// mbarrier + 1-D bulk-copy (TMA) staging, release/acquire flags, warp scans and
// the workspace error word.  Every wait here is bounded.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "si.h"

namespace si {

constexpr uint32_t kFullMask = 0xffffffffu;
// Every device-side wait gives up after this much wall time (read from
// %globaltimer) and records SI_ERR_TIMEOUT; legitimate waits last micro- to
// milliseconds.
constexpr uint64_t kWaitLimitNs = 4000000000ull;

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Deadline helper for a bounded wait: expired() becomes true `limit_ns`
// (default kWaitLimitNs) after construction.
struct WaitBudget {
    uint64_t start, limit;
    uint32_t polls = 0;
    __device__ __forceinline__ explicit WaitBudget(uint64_t limit_ns = kWaitLimitNs)
        : start(global_ns()), limit(limit_ns) {}
    __device__ __forceinline__ bool expired() {
        // the timer is read every 32 polls
        return ((++polls & 31u) == 0) && (global_ns() - start > limit);
    }
};

// ---------------------------------------------------------------- errors --
// The first words of every workspace: [0] error word (0 = ok, else si_status),
// [1] the site that recorded it, [2] a site-specific detail (e.g. a tile).
// [3] is the set of all sites that recorded an error (bit per site id < 32).
__device__ __forceinline__ void record_error(uint32_t* err, si_status code, uint32_t site = 0, uint32_t info = 0) {
    if (atomicCAS(err, 0u, static_cast<uint32_t>(code)) == 0u) {
        err[1] = site;
        err[2] = info;
    }
    atomicOr(err + 3, 1u << (site & 31u));
}

// --------------------------------------------------------------- smem/PTX --
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory load by 32-bit shared-window byte address.
__device__ __forceinline__ uint32_t lds_u32(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr));
    return v;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes an mbarrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// As mbar_try_wait, but the warp may be suspended (issuing nothing) for up to
// `hint_ns` while the phase is still open; it resumes as soon as the phase
// completes.
__device__ __forceinline__ bool mbar_try_wait_suspend(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return done != 0;
}

// Suspension hint of one poll of a bounded wait: long enough that a waiting
// warp takes no issue slots from the working ones, short against the budget.
constexpr uint32_t kSuspendHintNs = 1u << 20;

// Bounded wait on an mbarrier phase; records SI_ERR_TIMEOUT and returns false
// if it gives up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t* err, uint32_t site = 0,
                                                  uint32_t info = 0, uint64_t limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    WaitBudget budget(limit_ns);
    while (!budget.expired()) {
        if (mbar_try_wait_suspend(bar, parity, kSuspendHintNs)) return true;
    }
    record_error(err, SI_ERR_TIMEOUT, site, info);
    return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before its
// later async-proxy (bulk copy) ones.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Named barrier over `count` threads (id 0 is __syncthreads).
__device__ __forceinline__ void named_barrier(uint32_t id, uint32_t count) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Named barrier that also ORs a predicate over the `count` threads: every
// thread gets true if any passed true.
__device__ __forceinline__ bool named_barrier_or(uint32_t id, uint32_t count, bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "barrier.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"(v ? 1u : 0u), "r"(id), "r"(count)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ uint64_t ld_acquire_shared_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.acquire.cta.shared::cta.u64 %0, [%1];" : "=l"(v) : "r"(smem_addr(p)) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_shared_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.release.cta.shared::cta.u64 [%0], %1;" ::"r"(smem_addr(p)), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t ld_acquire_shared_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.cta.shared::cta.u32 %0, [%1];" : "=r"(v) : "r"(smem_addr(p)) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_shared_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.cta.shared::cta.u32 [%0], %1;" ::"r"(smem_addr(p)), "r"(v) : "memory");
}

// 1-D bulk copy global -> shared (TMA engine), completion counted on `bar`.
// dst and src must be 16-byte aligned and bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// ------------------------------------------------------- flags (look-back) --
__device__ __forceinline__ uint64_t ld_acquire_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Relaxed (unordered) 64-bit accesses at GPU scope: for status words whose
// flag and value travel together in one word, so no other access needs to be
// ordered with them.
__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// ------------------------------------------------------------ warp scans --
__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t n = __shfl_up_sync(kFullMask, v, d);
        if (lane >= d) v += n;
    }
    return v;
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(kFullMask, v, d);
    return v;
}

// ------------------------------------------------------ staging planning --
// Plan for copying n uint32 from global g into a 16-byte aligned shared
// buffer `buf` (capacity >= n + 8) so that element x lands at dst[x]:
// the 16-byte aligned middle goes through the bulk-copy engine, the <= 3
// leading and <= 3 trailing elements through ordinary loads.
struct StagePlan {
    uint32_t* dst;   // shared address of element 0
    int head;        // elements [0, head) by plain loads
    int body;        // elements [head, head + body) by bulk copy (body % 4 == 0)
    int n;           // elements [head + body, n) by plain loads
};

__device__ __forceinline__ StagePlan plan_stage(const uint32_t* g, int n, uint32_t* buf) {
    StagePlan p;
    const int mis = static_cast<int>((reinterpret_cast<uintptr_t>(g) & 15u) >> 2);
    int head = mis ? 4 - mis : 0;
    if (head > n) head = n;
    p.head = head;
    p.body = ((n - head) >> 2) << 2;
    p.dst = buf + ((4 - head) & 3);
    p.n = n;
    return p;
}

// Issued by one thread: the bulk part of a plan.
__device__ __forceinline__ void issue_stage(const StagePlan& p, const uint32_t* g, uint64_t* bar) {
    if (p.body > 0) bulk_g2s(p.dst + p.head, g + p.head, static_cast<uint32_t>(p.body) * 4u, bar);
}

// Done by threads [0, 6): the plain-load edges of a plan.
__device__ __forceinline__ void edge_stage(const StagePlan& p, const uint32_t* g, int slot) {
    int x = slot < 3 ? slot : p.head + p.body + (slot - 3);
    bool want = slot < 3 ? (slot < p.head) : (x < p.n);
    if (want) p.dst[x] = __ldg(g + x);
}

}  // namespace si
