// kw_fft.cuh — shared-memory Stockham FFT for sm_100a.
//
// A complex transform of length n = R_0 R_1 ... R_{s-1} runs as s radix stages. Stage t with
// Ns = R_0...R_{t-1} takes butterfly j in [0, n/R) from x[j + r n/R] (r < R), multiplies
// input r by exp(-+2 pi i r k / (Ns R)) with k = j mod Ns, does a length-R DFT in registers and
// writes y[(j - k) R + k + r Ns] (the self-sorting Stockham order; no bit reversal). Stages
// ping-pong between two shared-memory buffers. Twiddles are precomputed in FP64 on the host and
// rounded to FP32 (Engine::build_plan in kw_engine.cpp). Butterflies of radix 2, 3, 4, 5, 8, 12
// and 16 are unrolled in registers; any other prime radix runs through a direct O(R^2) DFT with
// FP64-derived roots.
#pragma once

#include "kw_common.h"

namespace kw {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse): the sign of the DFT kernel exp(-+ i pi/2)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
template <bool INV>
__device__ __forceinline__ float2 twiddle(float2 a, float2 w) { return INV ? cmulc(a, w) : cmul(a, w); }

// ---- in-register DFTs ---------------------------------------------------------------------
template <bool INV>
__device__ __forceinline__ void dft2(float2& a, float2& b) {
    float2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
    float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
    float2 s13 = cadd(a1, a3), d13 = mul_mi<INV>(csub(a1, a3));
    a0 = cadd(s02, s13);
    a2 = csub(s02, s13);
    a1 = cadd(d02, d13);
    a3 = csub(d02, d13);
}

template <int R, bool INV>
struct DFT;

template <bool INV>
struct DFT<2, INV> {
    __device__ __forceinline__ static void run(float2* v) { dft2<INV>(v[0], v[1]); }
};

template <bool INV>
struct DFT<4, INV> {
    __device__ __forceinline__ static void run(float2* v) { dft4<INV>(v[0], v[1], v[2], v[3]); }
};

template <bool INV>
struct DFT<3, INV> {
    __device__ __forceinline__ static void run(float2* v) {
        const float h = 0.86602540378443864676f;  // sin(2 pi / 3)
        float2 t = cadd(v[1], v[2]);
        float2 m = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
        float2 d = mul_mi<INV>(csub(v[1], v[2]));  // -+ i (a1 - a2)
        v[0] = cadd(v[0], t);
        v[1] = make_float2(m.x + h * d.x, m.y + h * d.y);
        v[2] = make_float2(m.x - h * d.x, m.y - h * d.y);
    }
};

template <bool INV>
struct DFT<5, INV> {
    __device__ __forceinline__ static void run(float2* v) {
        const float c1 = 0.30901699437494742410f;   // cos(2 pi/5)
        const float c2 = -0.80901699437494742410f;  // cos(4 pi/5)
        const float s1 = 0.95105651629515357212f;   // sin(2 pi/5)
        const float s2 = 0.58778525229247312917f;   // sin(4 pi/5)
        float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        float2 a0 = v[0];
        float2 b1 = make_float2(a0.x + c1 * t1.x + c2 * t2.x, a0.y + c1 * t1.y + c2 * t2.y);
        float2 b2 = make_float2(a0.x + c2 * t1.x + c1 * t2.x, a0.y + c2 * t1.y + c1 * t2.y);
        float2 e1 = mul_mi<INV>(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
        float2 e2 = mul_mi<INV>(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
        v[0] = cadd(a0, cadd(t1, t2));
        v[1] = cadd(b1, e1);
        v[4] = csub(b1, e1);
        v[2] = cadd(b2, e2);
        v[3] = csub(b2, e2);
    }
};

template <bool INV>
struct DFT<8, INV> {
    __device__ __forceinline__ static void run(float2* v) {
        const float r = 0.70710678118654752440f;
        float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
        float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        dft4<INV>(e0, e1, e2, e3);
        dft4<INV>(o0, o1, o2, o3);
        // o_k *= exp(-+ 2 pi i k / 8)
        o1 = INV ? make_float2(r * (o1.x - o1.y), r * (o1.x + o1.y)) : make_float2(r * (o1.x + o1.y), r * (o1.y - o1.x));
        o2 = mul_mi<INV>(o2);
        o3 = INV ? make_float2(-r * (o3.x + o3.y), r * (o3.x - o3.y)) : make_float2(r * (o3.y - o3.x), -r * (o3.x + o3.y));
        v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
        v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
        v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
        v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
    }
};

// 12 = 3 x 4: DFT4 over n2 for each n1 (x[n1 + 3 n2]), twiddle W12^{n1 k2}, DFT3 over n1 for each
// k2; output k2 + 4 k1.
template <bool INV>
struct DFT<12, INV> {
    __device__ __forceinline__ static void run(float2* v) {
        const float h = 0.86602540378443864676f;  // sqrt(3) / 2
        float2 y[3][4];
#pragma unroll
        for (int n1 = 0; n1 < 3; ++n1) {
#pragma unroll
            for (int n2 = 0; n2 < 4; ++n2) y[n1][n2] = v[n1 + 3 * n2];
            dft4<INV>(y[n1][0], y[n1][1], y[n1][2], y[n1][3]);
        }
        // exp(-2 pi i m / 12) for m = n1 k2: m = 1, 2, 3 (n1 = 1) and 2, 4, 6 (n1 = 2)
        const float2 w1 = make_float2(h, -0.5f), w2 = make_float2(0.5f, -h), w3 = make_float2(0.f, -1.f);
        const float2 w4 = make_float2(-0.5f, -h), w6 = make_float2(-1.f, 0.f);
        y[1][1] = twiddle<INV>(y[1][1], w1);
        y[1][2] = twiddle<INV>(y[1][2], w2);
        y[1][3] = twiddle<INV>(y[1][3], w3);
        y[2][1] = twiddle<INV>(y[2][1], w2);
        y[2][2] = twiddle<INV>(y[2][2], w4);
        y[2][3] = twiddle<INV>(y[2][3], w6);
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) {
            float2 t[3] = {y[0][k2], y[1][k2], y[2][k2]};
            DFT<3, INV>::run(t);
#pragma unroll
            for (int k1 = 0; k1 < 3; ++k1) v[k2 + 4 * k1] = t[k1];
        }
    }
};

template <bool INV>
struct DFT<16, INV> {
    __device__ __forceinline__ static void run(float2* v) {
        float2 e[8], o[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) { e[i] = v[2 * i]; o[i] = v[2 * i + 1]; }
        DFT<8, INV>::run(e);
        DFT<8, INV>::run(o);
        // exp(-2 pi i k/16), k = 0..7
        const float C1 = 0.92387953251128675613f, S1 = 0.38268343236508977173f;
        const float R2 = 0.70710678118654752440f;
        const float2 w[8] = {make_float2(1.f, 0.f), make_float2(C1, -S1), make_float2(R2, -R2), make_float2(S1, -C1),
                             make_float2(0.f, -1.f), make_float2(-S1, -C1), make_float2(-R2, -R2), make_float2(-C1, -S1)};
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            float2 t = twiddle<INV>(o[k], w[k]);
            v[k] = cadd(e[k], t);
            v[k + 8] = csub(e[k], t);
        }
    }
};

// ---- one Stockham stage for one butterfly ---------------------------------------------------
template <int R, bool INV>
__device__ __forceinline__ void stage_bfly(const float2* __restrict__ in, float2* __restrict__ out, int ldi,
                                           int j, int nb, int Ns, const float2* __restrict__ tw) {
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = in[(j + r * nb) * ldi];
    const int k = j % Ns;
    if (Ns > 1) {
        const float2* t = tw + k * (R - 1);
#pragma unroll
        for (int r = 1; r < R; ++r) v[r] = twiddle<INV>(v[r], __ldg(t + r - 1));
    }
    DFT<R, INV>::run(v);
    const int base = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) out[(base + r * Ns) * ldi] = v[r];
}

// Any radix R: direct DFT, roots exp(-2 pi i m / R) from `gen`.
template <bool INV>
__device__ __forceinline__ void stage_bfly_generic(const float2* __restrict__ in, float2* __restrict__ out, int ldi,
                                                   int j, int nb, int Ns, int R, const float2* __restrict__ tw,
                                                   const float2* __restrict__ gen) {
    const int k = j % Ns;
    const int base = (j - k) * R + k;
    for (int s = 0; s < R; ++s) {
        float2 acc = make_float2(0.f, 0.f);
        for (int q = 0; q < R; ++q) {
            float2 x = in[(j + q * nb) * ldi];
            if (Ns > 1 && q > 0) x = twiddle<INV>(x, __ldg(tw + k * (R - 1) + q - 1));
            const int m = (q * s) % R;
            x = twiddle<INV>(x, __ldg(gen + m));
            acc = cadd(acc, x);
        }
        out[(base + s * Ns) * ldi] = acc;
    }
}

// Transform `nlines` lines of length pl.n held in shared memory; element i of line l lives at
// buf[l * ldl + i * ldi]. `lines_fastest` maps consecutive threads to consecutive lines (use it
// when the lines are interleaved, ldl == 1). Returns the buffer that holds the result.
template <bool INV>
__device__ float2* fft_lines(float2* a, float2* b, const FFTPlanDev& pl, int nlines, int ldl, int ldi,
                             bool lines_fastest) {
    const int n = pl.n;
    int Ns = 1;
    for (int s = 0; s < pl.nstages; ++s) {
        const int R = pl.radix[s];
        const int nb = n / R;
        const int total = nb * nlines;
        const float2* tw = pl.tw + pl.tw_off[s];
        for (int w = threadIdx.x; w < total; w += blockDim.x) {
            int l, j;
            if (lines_fastest) { l = w % nlines; j = w / nlines; }
            else { j = w % nb; l = w / nb; }
            const float2* in = a + l * ldl;
            float2* out = b + l * ldl;
            switch (R) {
                case 2: stage_bfly<2, INV>(in, out, ldi, j, nb, Ns, tw); break;
                case 3: stage_bfly<3, INV>(in, out, ldi, j, nb, Ns, tw); break;
                case 4: stage_bfly<4, INV>(in, out, ldi, j, nb, Ns, tw); break;
                case 5: stage_bfly<5, INV>(in, out, ldi, j, nb, Ns, tw); break;
                case 8: stage_bfly<8, INV>(in, out, ldi, j, nb, Ns, tw); break;
                case 16: stage_bfly<16, INV>(in, out, ldi, j, nb, Ns, tw); break;
                default: stage_bfly_generic<INV>(in, out, ldi, j, nb, Ns, R, tw, pl.gen + pl.gen_off[s]); break;
            }
        }
        __syncthreads();
        float2* t = a; a = b; b = t;
        Ns *= R;
    }
    return a;
}

}  // namespace kw

// ============================================================================================
// Compile-time specialised Stockham transform for the common line lengths N = 2^a 3^b 5^c.
// The radix sequence, the number of lines per CTA (L) and every index are template constants,
// so a butterfly costs only its loads, twiddles, DFT and stores. One twiddle table per length
// (W_N^m = exp(-2 pi i m / N), m < N, FP64 rounded to FP32) serves every stage:
// exp(-2 pi i r k / (Ns R)) = W_N^{r k N / (Ns R)}.
// ============================================================================================
namespace kw {

// radix sequence: greedy 16, 8, 4, 2, then 3, 5 (the host plan uses the same rule)
__host__ __device__ constexpr int radix_at(int n, int k) {
    const int order[6] = {16, 8, 4, 2, 3, 5};
    int m = n, idx = 0;
    for (int oi = 0; oi < 6; ++oi) {
        const int r = order[oi];
        while (m % r == 0 && m > 1) {
            if (idx == k) return r;
            ++idx;
            m /= r;
        }
    }
    return 1;
}

__host__ __device__ constexpr bool fixed_fft_length(int n) {
    if (n < 2) return false;
    int m = n;
    while (m % 2 == 0) m /= 2;
    while (m % 3 == 0) m /= 3;
    while (m % 5 == 0) m /= 5;
    return m == 1;
}

// One in-place Stockham stage: every thread first gathers, twiddles and transforms all of its
// butterflies in registers, the block synchronises, then every thread scatters its results into
// the same buffer. One shared buffer per tile instead of two.
template <int N, int R, int Ns, int L, int LDI, bool INV>
__device__ __forceinline__ void tstage_inplace(float2* __restrict__ buf, const float2* __restrict__ twn, int nl) {
    constexpr int NB = N / R;
    constexpr int TPL = 256 / L;                 // threads per line
    constexpr int BPT = (NB + TPL - 1) / TPL;    // butterflies per thread
    const int l = threadIdx.x % L;
    const int j0 = threadIdx.x / L;
    const bool active = l < nl;
    float2 v[BPT][R];
#pragma unroll
    for (int b = 0; b < BPT; ++b) {
        const int j = j0 + b * TPL;
        if (active && j < NB) {
#pragma unroll
            for (int r = 0; r < R; ++r) v[b][r] = buf[(j + r * NB) * LDI + l];
            const int k = j % Ns;
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) v[b][r] = twiddle<INV>(v[b][r], __ldg(twn + r * k * (N / (Ns * R))));
            }
            DFT<R, INV>::run(v[b]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < BPT; ++b) {
        const int j = j0 + b * TPL;
        if (active && j < NB) {
            const int k = j % Ns;
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) buf[(base + r * Ns) * LDI + l] = v[b][r];
        }
    }
    __syncthreads();
}

template <int N, int S, int Ns, int L, int LDI, bool INV>
struct TStages {
    __device__ __forceinline__ static void run(float2* buf, const float2* __restrict__ twn, int nl) {
        constexpr int R = radix_at(N, S);
        if constexpr (R > 1) {
            tstage_inplace<N, R, Ns, L, LDI, INV>(buf, twn, nl);
            TStages<N, S + 1, Ns * R, L, LDI, INV>::run(buf, twn, nl);
        }
    }
};

// Transform (in place) nl <= L interleaved lines of length N: element i of line l at
// buf[i * LDI + l]. The caller synchronises before (data staged); the call ends synchronised.
template <int N, int L, int LDI, bool INV>
__device__ __forceinline__ float2* fft_tile(float2* buf, float2* /*unused*/, const float2* __restrict__ twn, int nl) {
    TStages<N, 0, 1, L, LDI, INV>::run(buf, twn, nl);
    return buf;
}

}  // namespace kw
