// lgm_device.cuh -- device-side building blocks shared by the sm_100a kernels.
//
// Bulk (non-tensor, non-multicast) TMA copies into shared memory completed on
// an mbarrier, bounded waits that report a timeout instead of spinning
// forever, and the packed FP32x2 arithmetic of sm_100.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace lgm {

// Device error bits, OR-ed into the context's error word.
enum : unsigned {
    DEVERR_SOURCE_RANGE = 1u,   // a source site outside [0, volume)
    DEVERR_TARGET_RANGE = 2u,   // a target site outside [0, volume + 35)
    DEVERR_TIMEOUT = 4u,        // a bounded wait on an mbarrier ran out
    DEVERR_STATE = 8u,          // a kernel found inconsistent state
};

// Iterations of mbarrier.try_wait before a wait is declared stuck.  Each
// try_wait may suspend the thread for a hardware-defined interval, so this is
// far above any legitimate wait (a bulk copy of a few KB) and still ends.
constexpr int kWaitLimit = 1 << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Order this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (bulk copy) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

// 1-D bulk copy global -> shared, completion counted on `bar`.  Both
// addresses 16-byte aligned, bytes a multiple of 16 (checked by the callers'
// layouts: chunks are whole multiples of 32-byte records).
__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Plain arrival (no transaction count), release semantics at CTA scope.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
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

// Bounded wait for phase `parity` of `bar`.  Returns false (and raises
// DEVERR_TIMEOUT) when `limit` tries run out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, unsigned* err,
                                                  int limit = kWaitLimit) {
    for (int it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    atomicOr(err, DEVERR_TIMEOUT);
    return false;
}

// After a wait ran out: wait (bounded, no error raised) for the phases of
// the bulk copies a CTA still has in flight -- sequence numbers first .. last-1
// of a two-stage pipeline, stage g & 1, phase (g >> 1) & 1 -- so that no copy
// lands in shared memory after the CTA has left.  One thread calls it.
__device__ __forceinline__ void mbar_drain_stages(uint64_t* bars, uint32_t first, uint32_t last,
                                                  int limit = kWaitLimit) {
    for (uint32_t g = first; g < last; ++g) {
        const uint32_t parity = (g >> 1) & 1u;
        for (int it = 0; it < limit; ++it)
            if (mbar_try_wait(&bars[g & 1u], parity)) break;
    }
}

// The same for an S-stage ring: sequence number g uses stage g % S and
// phase (g / S) & 1.
__device__ __forceinline__ void mbar_drain_ring(uint64_t* bars, int S, uint32_t first,
                                                uint32_t last, int limit = kWaitLimit) {
    for (uint32_t g = first; g < last; ++g) {
        const uint32_t parity = (g / (uint32_t)S) & 1u;
        for (int it = 0; it < limit; ++it)
            if (mbar_try_wait(&bars[g % (uint32_t)S], parity)) break;
    }
}

// MUFU reciprocal square root (PTX rsqrt.approx.ftz.f32).  rsqrt(+0) = +inf,
// rsqrt(+inf) = +0.
__device__ __forceinline__ float rsqrt_mufu(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// acc += q * w if key < lim (unsigned): one compare, one predicated FFMA.
__device__ __forceinline__ void fma_if_below(float& acc, float q, float w, unsigned key,
                                             unsigned lim) {
    asm("{\n\t.reg .pred p;\n\t"
        "setp.lt.u32 p, %1, %2;\n\t"
        "@p fma.rn.f32 %0, %3, %4, %0;\n\t}"
        : "+f"(acc)
        : "r"(key), "r"(lim), "f"(q), "f"(w));
}

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// Programmatic dependent launch.  A kernel launched with the programmatic
// stream serialization attribute may be scheduled before the kernel ahead of
// it in the stream has finished; pdl_wait() blocks until that kernel has
// completed and its memory operations are visible (a no-op for a kernel
// launched without the attribute).  Every kernel of a call's chain calls it
// before its first global memory access.  pdl_trigger() lets the next kernel
// of the stream be scheduled once every CTA of this grid has called it (or
// exited); it changes when the next kernel starts waiting, never what it sees.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

}  // namespace lgm
