// kw_async.cuh — asynchronous-copy plumbing for the warp-specialised pass kernels (sm_100a):
// mbarriers, TMA tensor loads (cp.async.bulk.tensor, CTA-local, never multicast) and named
// barriers for the consumer warps. Every wait is bounded: after about a second it records an error
// code in a global flag and reports failure, so a kernel can finish instead of hanging.
#pragma once

#include <cuda.h>
#include <cstdint>

namespace kw {

// error codes a kernel leaves in the engine's error flag
enum KernelError { KE_NONE = 0, KE_TIMEOUT_FULL = 1, KE_TIMEOUT_EMPTY = 2, KE_TIMEOUT_DRAIN = 3 };

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// make the initialised barriers visible to the async (TMA) proxy
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_test_parity(uint64_t* bar, uint32_t parity) {
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

// default limit of a bounded wait: ~1.1 s at 1.9 GHz
constexpr long long kWaitCycles = 1LL << 31;

// Wait until the phase with the given parity has completed; false (and `err` set) after `limit`
// clock64 cycles.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code,
                                          long long limit = kWaitCycles) {
    if (mbar_test_parity(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_test_parity(bar, parity)) {
        if (clock64() - t0 > limit) {
            atomicCAS(err, 0, code);
            return false;
        }
    }
    return true;
}

// As mbar_wait, but also gives up (returning false without recording an error) once `*abort` is
// set: the producer of a pass whose consumers have stopped stops issuing copies at once.
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t* bar, uint32_t parity, int* err, int code,
                                                   const volatile int* abort) {
    if (mbar_test_parity(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_test_parity(bar, parity)) {
        if (*abort) return false;
        if (clock64() - t0 > kWaitCycles) {
            atomicCAS(err, 0, code);
            return false;
        }
    }
    return true;
}

// 2D / 3D tile loads from a tensor map in global memory into this CTA's shared memory, completing
// on `bar` (transaction bytes). Coordinates are element indices, innermost first.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// L2 prefetch of a tile through its tensor map: no shared memory and no completion to wait for
// (the same coordinate rules as the loads)
__device__ __forceinline__ void tma_prefetch_2d(const CUtensorMap* map, int x, int y) {
    asm volatile("cp.async.bulk.prefetch.tensor.2d.L2.global.tile [%0, {%1, %2}];"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y) : "memory");
}
__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap* map, int x, int y, int z) {
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z) : "memory");
}

// barrier among the first `nthreads` threads (the consumer warps) — id 0 is __syncthreads'
__device__ __forceinline__ void named_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

}  // namespace kw
