// kw_pass_common.cuh — shared pieces of the persistent, cp.async-pipelined pass kernels.
//
// Every pass kernel is instantiated per line length (a compile-time constant; 0 = runtime plan)
// and launched once per size class of the engine's simulations. A CTA walks its share of the
// launch's tile list with a two-stage pipeline: tile k+1 is copied HBM -> shared memory with
// cp.async while tile k is transformed on chip.
#pragma once

#include "kw_device.cuh"

#include <algorithm>

namespace kw {

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Stage `nrows` rows of `C` floats (row stride C) into dst (row-major, same stride).
__device__ __forceinline__ void stage_rows(float* dst, const float* src, int nrows, int C) {
    const int n = nrows * C;
    if ((C & 3) == 0 && ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) == 0) {
        for (int w = threadIdx.x * 4; w < n; w += blockDim.x * 4) cp_async16(dst + w, src + w);
    } else {
        for (int w = threadIdx.x; w < n; w += blockDim.x) cp_async4(dst + w, src + w);
    }
}

// Switch the CTA's cached descriptor to simulation `sim` (all threads call it).
__device__ __forceinline__ void use_sim(SimDev& S, int& cur, const SimDev* __restrict__ sims, int sim) {
    __syncthreads();
    if (sim != cur) {
        load_sim(S, sims + sim);
        __syncthreads();
        cur = sim;
    }
}


// persistent grid: as many CTAs as can be resident, at most one per tile
inline int persistent_grid(const void* fn, size_t smem, int nmap) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, smem) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    return std::max(1, std::min(nmap, per_sm * sms));
}

inline void set_max_smem(const void* fn, int optin) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) return;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

}  // namespace kw
