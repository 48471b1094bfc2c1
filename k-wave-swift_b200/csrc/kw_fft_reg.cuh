// kw_fft_reg.cuh — register-resident two-stage transform of N = R1 * R2 points (R1 >= R2).
//
// A line is handled by T = R2 threads of a CTA; thread t holds the R1 values x[t + T r] (r < R1).
//   stage 1  radix-R1 DFT in registers (butterfly j = t), outputs y[t R1 + r] to shared memory
//   stage 2  NB = R1 / R2 radix-R2 DFTs per thread (butterflies j2 = t + b T) on y[j2 + R1 r],
//            twiddled by W_N^{r j2}; output r of butterfly j2 is X[j2 + R1 r] = X[t + T (b + NB r)]
// so on exit thread t holds X[t + T m] (m < R1) — the same ownership as on entry. A forward
// transform, a pointwise product and an inverse transform therefore chain in registers with one
// shared-memory exchange per transform.
//
// The shared-memory layout is a policy: Lay::at(j, l) is the slot of value j of line l.
#pragma once

#include "kw_fft.cuh"

namespace kw {

template <int N>
struct TwoStage {
    static constexpr int R1 = colr_r1(N);
    static constexpr int R2 = N / R1;
    static constexpr int T = R2;             // threads per line
    static constexpr int NB = R1 / R2;       // stage-2 butterflies per thread
    static constexpr int LINES = 256 / T;    // lines per 256-thread CTA
    static_assert(R1 >= R2 && R1 % R2 == 0 && T * LINES == 256, "two-stage split");
};

// Lines are consecutive lanes (column passes): slot j * LD + l. With LD = LINES + 1 a half-warp
// (16 consecutive lines, one j) touches 16 consecutive slots.
template <int N>
struct ColLayout {
    static constexpr int LD = TwoStage<N>::LINES + 1;
    static constexpr int SLOTS = N * LD;
    __device__ __forceinline__ static int at(int j, int l) { return j * LD + l; }
};

// Threads of one line are consecutive lanes (row passes, coalesced along the row): slot
// l * LDL + j + j / R1. The stage-1 stores (j = t R1 + r) then step R1 + 1 (odd) slots between
// lanes, the stage-2 loads (j = j2 + R1 r) step one slot, and LDL = T (R1 + 1) = N + T is
// congruent to T modulo 16, so the 16 / T lines of a half-warp land on disjoint banks.
template <int N>
struct RowLayout {
    static constexpr int R1 = TwoStage<N>::R1;
    static constexpr int LDL = TwoStage<N>::T * (R1 + 1);
    static constexpr int SLOTS = TwoStage<N>::LINES * LDL;
    __device__ __forceinline__ static int at(int j, int l) { return l * LDL + j + j / R1; }
};

template <int N, bool INV, class Lay>
struct FftReg {
    using P = TwoStage<N>;
    // v[m] = x[t + T m] on entry, X[t + T m] on exit (unnormalised). Every thread of the CTA
    // calls this together (two barriers); `sh` is free again on return.
    __device__ __forceinline__ static void run(float2 (&v)[P::R1], float2* sh, int t, int l,
                                               const float2* __restrict__ twn) {
        constexpr int R1 = P::R1, R2 = P::R2, T = P::T;
        DFT<R1, INV>::run(v);
#pragma unroll
        for (int r = 0; r < R1; ++r) sh[Lay::at(t * R1 + r, l)] = v[r];
        __syncthreads();
#pragma unroll
        for (int b = 0; b < P::NB; ++b) {
            const int j2 = t + b * T;
            float2 w[R2];
#pragma unroll
            for (int r = 0; r < R2; ++r) w[r] = sh[Lay::at(j2 + R1 * r, l)];
#pragma unroll
            for (int r = 1; r < R2; ++r) w[r] = twiddle<INV>(w[r], __ldg(twn + r * j2));
            DFT<R2, INV>::run(w);
#pragma unroll
            for (int r = 0; r < R2; ++r) v[b + r * P::NB] = w[r];
        }
        __syncthreads();
    }
};

}  // namespace kw
