// jw_async.cuh -- tensor-memory-accelerator (TMA) tile loads and the
// shared-memory barriers (mbarrier) that report their completion, for the
// persistent column pass of the mixed-precision step.
//
// A load is one cp.async.bulk.tensor.2d from global memory into this CTA's own
// shared memory (no cluster multicast), its completion counted in bytes on an
// mbarrier (complete_tx).  Every wait is bounded: a wait that runs out returns
// false, and the caller raises JW_FLAG_TIMEOUT and stops issuing work.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "jw_common.cuh"

namespace jw {

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// makes the initialised barriers visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// arrive (count 1) and expect `bytes` of transactions before the phase completes
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}

// Wait until the barrier's phase with this parity has completed, for at most
// ~limit_ns of wall time.  Returns false if the wait ran out.
// The clock is read only after 1024 unsuccessful tries, so that waits that end
// soon issue nothing but the tries.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity,
                                                  uint64_t limit_ns = 2000000000ull) {
    uint64_t t0 = 0;
    for (unsigned it = 0; it < (1u << 26); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 1023u) == 1023u) {
            const uint64_t t = global_ns();
            if (it == 1023u) t0 = t;
            else if (t - t0 > limit_ns) return false;
        }
    }
    return false;
}

// Orders this thread's earlier generic-proxy accesses of shared memory (and,
// after a CTA barrier, every thread's) before later TMA writes to it.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// 2D tile load: the box at element coordinates (x, y) of the tensor map into
// dst (this CTA's shared memory), completion counted on bar.  x * element
// size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];\n" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// 2D tile store: src (this CTA's shared memory, the box's dense layout) to
// the box at element coordinates (x, y) of the tensor map, as one bulk group
// of this thread (tma_store_commit).  Coordinates must be non-negative and
// x * element size a multiple of 16 bytes.
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, int x, int y, const void* src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(x), "r"(y), "r"(smem_addr(src))
                 : "memory");
}
__device__ __forceinline__ void tma_store_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's bulk store groups are still reading shared memory
template <int N>
__device__ __forceinline__ void tma_store_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;\n" ::"n"(N) : "memory");
}
// wait until at most N of this thread's bulk store groups are incomplete
template <int N>
__device__ __forceinline__ void tma_store_wait() {
    asm volatile("cp.async.bulk.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

}  // namespace jw
