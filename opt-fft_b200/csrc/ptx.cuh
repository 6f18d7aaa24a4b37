// ptx.cuh -- inline-PTX wrappers for sm_100a: mbarriers, bulk (TMA) copies,
// Ampere-style async copies, proxy fences, and bounded waits.
//
// Every wait here is bounded: after kSpinLimit polls it gives up and reports
// failure, so a lost completion turns into an error status read by the host
// instead of a hung GPU.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fft3d {

// Error codes written to a plan's device error word (first writer wins).
constexpr int DEV_ERR_NONE = 0;
constexpr int DEV_ERR_LOAD_TIMEOUT = 1;    // a stage load never completed
constexpr int DEV_ERR_CLUSTER_TIMEOUT = 2; // a cluster peer never arrived
constexpr int DEV_ERR_QUEUE_TIMEOUT = 3;   // a work-queue flag never became ready
constexpr int DEV_ERR_DEP_TIMEOUT = 4;     // a two-pass dependency counter never arrived

constexpr uint32_t kSpinLimit = 1u << 24;
// Wall-clock bound of a wait on a global counter that other CTAs advance.
constexpr unsigned long long kCounterWaitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Load with acquire semantics at GPU scope.
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Add with release semantics at GPU scope (no return value).
__device__ __forceinline__ void red_release_gpu_add(unsigned *p, unsigned v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Wait until *p >= target, or *abort becomes nonzero, or kCounterWaitNs pass.
// Returns true when the target was reached.  One thread calls it.
__device__ __forceinline__ bool wait_counter_geq(const unsigned *p, unsigned target,
                                                 const unsigned *abort)
{
    if (ld_acquire_gpu(p) >= target) return true;
    const unsigned long long t0 = globaltimer_ns();
    unsigned ns = 32;
    for (uint32_t i = 0; i < kSpinLimit; ++i) {
        __nanosleep(ns);
        if (ns < 1024) ns *= 2;
        if (ld_acquire_gpu(p) >= target) return true;
        if (ld_acquire_gpu(abort) != 0) return false;
        if (globaltimer_ns() - t0 > kCounterWaitNs) return false;
    }
    return false;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

// Make mbarrier initialisation visible to the async proxy (TMA) and the cluster.
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kSpinLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Order this thread's generic-proxy shared-memory accesses before later
// async-proxy (TMA) accesses of the same memory.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Order this thread's generic-proxy view of global memory (e.g. an acquire that
// found another CTA's data published) before its later async-proxy (TMA) reads.
__device__ __forceinline__ void fence_proxy_async_global()
{
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

// One-dimensional bulk copy global -> shared (TMA, no tensor map), completing
// `bytes` of transaction count on `bar`.  dst, src 16-byte aligned; bytes % 16 == 0.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// L2 eviction-priority policies for cache-hinted accesses: evict_first for
// data read or written once, evict_last for data that should stay in L2.
__device__ __forceinline__ uint64_t l2_policy_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ uint64_t l2_policy_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// bulk_g2s with an L2 cache policy for the source lines.
__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                              uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// One-dimensional bulk copy shared -> global (TMA, no tensor map) in this
// thread's current bulk group.  dst, src 16-byte aligned; bytes % 16 == 0.
__device__ __forceinline__ void bulk_s2g(void *dst, const void *src, uint32_t bytes)
{
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst),
                 "r"(smem_u32(src)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit()
{
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// Wait until at most N of this thread's bulk groups still read their shared-memory
// source (the source may then be overwritten).
template <int N>
__device__ __forceinline__ void bulk_wait_read()
{
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// Wait until at most N of this thread's bulk groups are incomplete (their
// writes performed).
template <int N>
__device__ __forceinline__ void bulk_wait()
{
    asm volatile("cp.async.bulk.wait_group %0;" ::"n"(N) : "memory");
}

// L2-only stores of one complex value with an L2 cache policy.
__device__ __forceinline__ void st_cg_hint(double2 *p, double2 v, uint64_t policy)
{
    asm volatile("st.global.cg.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(v.x), "d"(v.y),
                 "l"(policy)
                 : "memory");
}

__device__ __forceinline__ void st_cg_hint(float2 *p, float2 v, uint64_t policy)
{
    asm volatile("st.global.cg.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(v.x), "f"(v.y),
                 "l"(policy)
                 : "memory");
}

// Drop the 128-byte L2 line at p (128-byte aligned) without writing it back;
// its contents become undefined.  For scratch read for the last time, so that
// its dirty lines never reach HBM.
__device__ __forceinline__ void discard_l2_line(uintptr_t p)
{
    asm volatile("discard.global.L2 [%0], 128;" ::"l"(p) : "memory");
}

// Per-thread asynchronous copies global -> shared (cp.async, 16 or 8 bytes).
__device__ __forceinline__ void cp_async_16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
}

__device__ __forceinline__ void cp_async_8(void *dst, const void *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;" ::: "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ------------------------------------------------------------------ clusters

__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// Hardware cluster barrier; used once after mbarrier initialisation, when every
// CTA of the cluster is resident by the launch guarantee.
__device__ __forceinline__ void cluster_sync_hw()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::
                     : "memory");
}

// Shared-memory address (32-bit, shared::cluster window) of `p` in CTA `rank`.
__device__ __forceinline__ uint32_t mapa_u32(const void *p, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(p)), "r"(rank));
    return r;
}

// Arrive (release, cluster scope) on the mbarrier at a shared::cluster address.
__device__ __forceinline__ void mbar_arrive_remote(uint32_t cluster_addr)
{
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(cluster_addr)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait, acquire at cluster scope (pairs with mbar_arrive_remote).
__device__ __forceinline__ bool mbar_wait_cluster_bounded(uint64_t *bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kSpinLimit; ++i)
        if (mbar_try_wait_cluster(bar, parity)) return true;
    return false;
}

// Loads from another CTA's shared memory (shared::cluster address).
__device__ __forceinline__ double2 ld_dsmem_f64x2(uint32_t addr)
{
    double2 v;
    asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"(addr)
                 : "memory");
    return v;
}

__device__ __forceinline__ float2 ld_dsmem_f32x2(uint32_t addr)
{
    float2 v;
    asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr)
                 : "memory");
    return v;
}

// Record the first device-side error of a launch.
__device__ __forceinline__ void report_error(int *err, int code)
{
    if (err) atomicCAS(err, 0, code);
}

// Programmatic dependent launch.  A kernel launched with the programmatic
// stream-serialization attribute may have its CTAs placed while the previous
// kernel of the stream drains; griddepcontrol.wait then blocks until that
// kernel has completed and its memory operations are visible, so everything
// after it may read the previous kernel's output and overwrite its input.
// Without the attribute the wait returns at once.  launch_dependents lets the
// next such kernel place its CTAs as ours exit.  Called first in every kernel
// that launch_entry starts, before any global memory access.
__device__ __forceinline__ void pdl_begin()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

}  // namespace fft3d
