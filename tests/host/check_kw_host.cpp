// Host-side helpers of the engine (k-wave-swift_b200/csrc/kw_host.h), checked without a GPU:
// parallel_for visits every index once; flat_nonzero equals the sequential mask scan; and
// transpose_series turns the device's [T][np] sensor rows into the [np][T] output exactly as the
// element-by-element loop does, on the serial (small) and threaded (large) paths and for sensor
// counts that are not multiples of the block.
#include "kw_host.h"

#include <cstdio>
#include <random>

int main() {
    std::mt19937 rng(7);
    const size_t cases[][2] = {{1, 1}, {3, 5}, {7, 63}, {5, 64}, {9, 65}, {201, 224}, {300, 4099}, {1117, 2049}, {33, 100001}};
    for (const auto& c : cases) {
        const size_t T = c[0], np = c[1];
        std::vector<float> src(T * np), got(T * np, -1.f), want(T * np, -2.f);
        for (auto& x : src) x = (float)(rng() % 100000) * 0.5f;
        kw::transpose_series(src.data(), got.data(), T, np);
        for (size_t q = 0; q < np; ++q)
            for (size_t t = 0; t < T; ++t) want[q * T + t] = src[t * np + q];
        if (got != want) {
            std::printf("transpose_series mismatch at T=%zu np=%zu\n", T, np);
            return 1;
        }
    }
    for (long long n : {0LL, 1LL, 1000LL, 65536LL, 200003LL}) {
        std::vector<int> hits((size_t)n, 0);
        kw::parallel_for(n, [&](long long i) { hits[(size_t)i] += 1; });
        for (int h : hits)
            if (h != 1) {
                std::printf("parallel_for coverage wrong for n=%lld\n", n);
                return 1;
            }
    }
    // flat_nonzero: chunked counts + offsets give the sequential scan's ascending indices
    for (long long n : {0LL, 1LL, 17LL, 262144LL, 262145LL, 1000003LL}) {
        for (int density : {0, 1, 50, 100}) {
            std::vector<float> mask((size_t)n, 0.f);
            for (auto& x : mask) x = (int)(rng() % 100) < density ? 1.f : 0.f;
            std::vector<int> want;
            for (long long i = 0; i < n; ++i)
                if (mask[(size_t)i] != 0.0f) want.push_back((int)i);
            if (kw::flat_nonzero(mask.data(), n) != want) {
                std::printf("flat_nonzero mismatch for n=%lld density=%d\n", n, density);
                return 1;
            }
        }
    }
    std::printf("ok\n");
    return 0;
}
