// kw_host.h — host-side helpers of the engine: a parallel loop over the host's cores and the
// sensor-series transpose of the output copy.
#pragma once

#include <algorithm>
#include <cstddef>
#include <thread>
#include <vector>

namespace kw {

// fn(i) for i in [0, n) on the host's cores (at most 32 threads), or on the calling thread when n
// is below `min_parallel`. Callers pass functions of the index alone, writing disjoint outputs, so
// the split changes no value.
template <typename F>
void parallel_for(long long n, F&& fn, long long min_parallel = 1LL << 16) {
    const long long nt = std::min<long long>(std::max(1u, std::thread::hardware_concurrency()), 32);
    if (n < min_parallel || nt == 1 || n < 2) {
        for (long long i = 0; i < n; ++i) fn(i);
        return;
    }
    std::vector<std::thread> pool;
    const long long chunk = (n + nt - 1) / nt;
    for (long long k = 0; k < nt; ++k) {
        const long long lo = k * chunk, hi = std::min(n, lo + chunk);
        if (lo >= hi) break;
        pool.emplace_back([lo, hi, &fn] {
            for (long long i = lo; i < hi; ++i) fn(i);
        });
    }
    for (auto& t : pool) t.join();
}

// Sensor series: the device keeps [T][np] (one row per time step, written by the per-step gather);
// the output is [np][T] row-major (SimulationOutput's [nSensor, nt]). Blocks of 64 sensors: each
// time step's 64 values are read as one contiguous run and written to the block's 64 output rows,
// whose cache lines stay resident while t advances. Blocks go to the host's cores.
inline void transpose_series(const float* src, float* dst, size_t T, size_t np) {
    constexpr size_t QB = 64;
    const long long nblk = (long long)((np + QB - 1) / QB);
    const long long min_parallel = (T * np >= ((size_t)1 << 20)) ? 2 : (1LL << 62);
    parallel_for(nblk, [&](long long b) {
        const size_t q0 = (size_t)b * QB, q1 = std::min(np, q0 + QB);
        for (size_t t = 0; t < T; ++t) {
            const float* row = src + t * np;
            for (size_t q = q0; q < q1; ++q) dst[q * T + t] = row[q];
        }
    }, min_parallel);
}

// Ascending flat indices of the non-zero entries of a mask (flatNonzeroIndices, KSFO:778-782):
// the order of sensor points and source rows. Chunks are counted on the host's cores, then each
// chunk writes its indices at its offset, so the result equals the sequential scan.
inline std::vector<int> flat_nonzero(const float* m, long long n) {
    constexpr long long CH = 1LL << 18;
    const long long nch = (n + CH - 1) / CH;
    std::vector<long long> cnt((size_t)nch + 1, 0);
    parallel_for(nch, [&](long long c) {
        long long k = 0;
        for (long long i = c * CH, e = std::min(n, i + CH); i < e; ++i) k += m[i] != 0.0f;
        cnt[(size_t)c + 1] = k;
    }, 2);
    for (long long c = 0; c < nch; ++c) cnt[(size_t)c + 1] += cnt[(size_t)c];
    std::vector<int> r((size_t)cnt[(size_t)nch]);
    parallel_for(nch, [&](long long c) {
        long long o = cnt[(size_t)c];
        for (long long i = c * CH, e = std::min(n, i + CH); i < e; ++i)
            if (m[i] != 0.0f) r[(size_t)o++] = (int)i;
    }, 2);
    return r;
}

}  // namespace kw
