// kw_fft_reg.cuh — register-resident Stockham transform of N = R1 * R_1 * ... * R_last points
// (every later radix divides R1: powers of two with R1 = 4, 8 or 16, and 12 * 2^k with R1 = 12).
//
// A line is handled by T = N / R1 threads; thread t holds the R1 values x[t + T r] (r < R1).
//   stage 0   radix-R1 DFT in registers (butterfly j = t); outputs y[t R1 + r] to shared memory
//   stage s   radix R (R divides R1), Ns = product of the earlier radices: every thread runs
//             NB = R1 / R butterflies j = t + b T on y[j + r N / R], twiddled by W_{Ns R}^{(j mod Ns) r};
//             output r goes to y[(j / Ns) Ns R + (j mod Ns) + r Ns]
//   last      the outputs stay in registers: output r of butterfly j = t + b T is
//             X[j + r N / R] = X[t + T (b + NB r)]
// so on exit thread t holds X[t + T m] (m < R1) — the same ownership as on entry. A forward
// transform, a pointwise product and an inverse transform therefore chain in registers.
//
// The shared-memory layout is a policy: Lay::at(j, l) is the slot of value j of line l.
#pragma once

#include "kw_fft.cuh"

namespace kw {

template <int N, int R1_>
struct RegPlan {
    static constexpr int R1 = R1_;
    static constexpr int T = N / R1;           // threads per line
    static constexpr int LINES = 256 / T;      // lines per 256 threads
    __host__ __device__ static constexpr int gcd(int a, int b) { return b == 0 ? a : gcd(b, a % b); }
    // radix of stage s: R1 for stage 0, then the largest divisor of R1 that divides what is left
    // (every later radix divides R1, so each thread runs a whole number of butterflies)
    __host__ __device__ static constexpr int radix(int s) {
        int left = N / R1;
        int r = R1;
        for (int i = 1; i <= s; ++i) {
            r = gcd(R1, left);
            left /= r;
        }
        return r;
    }
    __host__ __device__ static constexpr int before(int s) {   // Ns: product of the radices of stages < s
        int p = 1;
        for (int i = 0; i < s; ++i) p *= radix(i);
        return p;
    }
    __host__ __device__ static constexpr int stages() {
        int n = 0;
        while (n < 32 && before(n) < N && radix(n) > 1) ++n;
        return n;
    }
    static constexpr int NSTAGES = stages();
    static_assert(N % R1 == 0 && T >= 1 && T <= 256 && 256 % T == 0, "register plan");
    static_assert(before(NSTAGES) == N && NSTAGES >= 2, "register plan stages");
};

// Lines are consecutive lanes (column passes): slot j * LD + l with LD = LINES + 1.
template <class P, int N>
struct ColLayout {
    static constexpr int LD = P::LINES + 1;
    static constexpr int SLOTS = N * LD;
    __device__ __forceinline__ static int at(int j, int l) { return j * LD + l; }
};

// Threads of one line are consecutive lanes (row passes, coalesced along the row): slot
// l * LDL + j + j / R1. Stage-0 stores (j = t R1 + r) then step R1 + 1 (odd) slots between lanes,
// later stages mostly one slot, and LDL = T (R1 + 1) = N + T is congruent to T modulo 16, so the
// 16 / T lines of a half-warp land on different banks.
template <class P, int N>
struct RowLayout {
    static constexpr int LDL = P::T * (P::R1 + 1);
    static constexpr int SLOTS = P::LINES * LDL;
    __device__ __forceinline__ static int at(int j, int l) { return l * LDL + j + j / P::R1; }
};

// Barrier policies: the whole CTA, or the 256 consumer threads of a warp-specialised CTA (named
// barrier 1; the producer warp does not take part).
struct BlockSync {
    __device__ __forceinline__ static void sync() { __syncthreads(); }
};
struct ConsumerSync {
    __device__ __forceinline__ static void sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }
};

template <int N, class P, bool INV, class Lay, class Sync, int S>
struct RegStage {
    __device__ __forceinline__ static void run(float2 (&v)[P::R1], float2* sh, int t, int l,
                                               const float2* __restrict__ twn) {
        constexpr int R1 = P::R1, T = P::T;
        constexpr int R = P::radix(S), Ns = P::before(S), NB = R1 / R;
        constexpr bool LAST = S == P::NSTAGES - 1;
        constexpr int TWSTEP = N / (Ns * R);
        float2 w[NB][R];
#pragma unroll
        for (int b = 0; b < NB; ++b)
#pragma unroll
            for (int r = 0; r < R; ++r) w[b][r] = sh[Lay::at(t + b * T + r * (N / R), l)];
        if (!LAST) Sync::sync();   // every input is read before any output overwrites it
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = t + b * T;
            const int k = j % Ns;
#pragma unroll
            for (int r = 1; r < R; ++r) w[b][r] = twiddle<INV>(w[b][r], __ldg(twn + k * r * TWSTEP));
            DFT<R, INV>::run(w[b]);
            if (LAST) {
#pragma unroll
                for (int r = 0; r < R; ++r) v[b + r * NB] = w[b][r];
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) sh[Lay::at((j / Ns) * Ns * R + k + r * Ns, l)] = w[b][r];
            }
        }
        Sync::sync();
        if constexpr (!LAST) RegStage<N, P, INV, Lay, Sync, S + 1>::run(v, sh, t, l, twn);
    }
};

template <int N, class P, bool INV, class Lay, class Sync = BlockSync>
struct FftReg {
    // v[m] = x[t + T m] on entry, X[t + T m] on exit (unnormalised). Every thread of the barrier
    // group calls this together; `sh` (Lay::SLOTS values) is free again on return.
    __device__ __forceinline__ static void run(float2 (&v)[P::R1], float2* sh, int t, int l,
                                               const float2* __restrict__ twn) {
        DFT<P::R1, INV>::run(v);
#pragma unroll
        for (int r = 0; r < P::R1; ++r) sh[Lay::at(t * P::R1 + r, l)] = v[r];
        Sync::sync();
        RegStage<N, P, INV, Lay, Sync, 1>::run(v, sh, t, l, twn);
    }
};

}  // namespace kw
