// kw_pass_rowr.cu — register-resident row passes for even rows whose half length M = C / 2 has a
// register plan (has_reg_row: powers of two 16 ... 2048 and 12 * 2^k up to 1536).
//
// A 256-thread CTA owns 256 / T consecutive rows; the T threads of a row are consecutive lanes, so
// every load and store walks the row contiguously. Thread t of a row holds the packed values
// z[t + T m] = x[2n] + i x[2n+1] (n = t + T m) of the M-point transform in registers
// (kw_fft_reg.cuh), i.e. the real samples 2n and 2n+1, which is also the pair its epilogue updates.
//
//   R2C   load the real row as float2 -> forward transform -> Hermitian split into X[0 .. M]
//   C2R   load X[k] and X[M-k] -> Hermitian merge -> inverse transform -> fused physics update
//
// Coupled epilogues (density: one spectrum per axis; power law: two) transform their components
// one after the other in the same CTA and park the finished ones in shared memory (each thread its
// own slots). The epilogue reads its field inputs for a few pairs at a time before any store, so
// their latencies overlap.
#include <cstdlib>

#include "kw_adjoint.h"
#include "kw_fft_reg.cuh"
#include "kw_pass_common.cuh"

namespace kw {

// ---------------------------------------------------------------------------------------------
// R2C: X[k] = (Z[k] + conj Z[M-k]) / 2 - i W_C^k (Z[k] - conj Z[M-k]) / 2, k = 0 .. M
// ---------------------------------------------------------------------------------------------
// Resident CTAs per SM the register budget of a C2R kernel is cut to (3 = at most 85 registers a
// thread): the epilogues that fit without spilling take three CTAs per SM for more loads in flight;
// the others, and the R2C, keep the compiler's choice (0: no minimum; a minimum of 1 lets the compiler
// take more registers and the 384-point rows ran 1.4x slower with it).
template <int M, int EPI, bool TAPE, int VAR = 0>
constexpr int rowr_minb() {
    // VAR bit 1 swaps two and three CTAs per SM for rows up to 128 (launch-shape variants)
    if (VAR & 2) return M <= 128 ? (rowr_minb<M, EPI, TAPE, 0>() == 3 ? 2 : 3) : rowr_minb<M, EPI, TAPE, 0>();
    // left alone these take 129-152 registers at some lengths (one CTA per SM)
    if (EPI == EPI_ADJ_EOS || EPI == EPI_ADJ_EOS_RHO || EPI == EPI_ADD_RHO || TAPE || M >= 768) return 2;
    // the density update with the precorrected source reads one field more: two CTAs per SM above
    // 128-point rows; up to 128, three with one pair of inputs in flight per batch (measured at
    // 256^3: 0.238 ms against 0.273 ms for two CTAs per SM with two pairs)
    if (EPI == EPI_DEN_SRC) return M <= 128 ? 3 : 2;
    return M <= 128 ? 3 : 0;
}

// one bin of the split, zk = Z[k], zm = Z[M - k], w = W_C^k
__device__ __forceinline__ float2 r2c_bin(float2 zk, float2 zm, float2 w) {
    const float2 E = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 D = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y + zm.y));
    const float2 O = make_float2(D.y, -D.x);   // -i D
    return cadd(E, cmul(O, w));
}

// Forward transform of the packed real row in v (z[t + T m]) and its Hermitian split into row
// `out` of a half spectrum. Every thread of the CTA calls it (the split reads Z[M - k] from another
// thread through `sh`); threads of rows past the end (ok = false) take part in the barriers only.
// `sh` is free again on return.
template <int M, class P, class Lay>
__device__ __forceinline__ void rowr_forward(float2 (&v)[P::R1], float2* sh, int t, int l, const float2* __restrict__ twn,
                                             const float2* __restrict__ tw, float2* out, bool ok) {
    constexpr int R1 = P::R1, T = P::T;
    FftReg<M, P, false, Lay>::run(v, sh, t, l, twn);
#pragma unroll
    for (int m = 0; m < R1; ++m) sh[Lay::at(t + T * m, l)] = v[m];
    __syncthreads();
    if (ok) {
#pragma unroll
        for (int m = 0; m < R1; ++m) {
            const int k = t + T * m;
            out[k] = r2c_bin(v[m], sh[Lay::at(k == 0 ? 0 : M - k, l)], __ldg(tw + k));
        }
        if (t == 0) out[M] = r2c_bin(v[0], v[0], __ldg(tw + M));
    }
    __syncthreads();
}

template <int M>
__global__ void __launch_bounds__(256) k_rowr_r2c(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                                  const BlockWork* __restrict__ map, int nmap, RowR2CJob job) {
    pdl_enter();
    using P = RegPlan<M, reg_r1(M)>;
    using Lay = RowLayout<P, M>;
    constexpr int R1 = P::R1, T = P::T, TW = P::LINES;
    __shared__ float2 sh[Lay::SLOTS];
    if (blockIdx.x >= nmap) return;
    const BlockWork bw = map[blockIdx.x];
    const SimDev& S = sims[bw.sim];
    if (!gate_open(S, job.gate, bw.comp, *d_t)) return;
    const int t = threadIdx.x % T, l = threadIdx.x / T;
    const int row = bw.tile * TW + l;
    const bool ok = row < S.A * S.B;
    if (job.ahead > 0 && threadIdx.x == 0 && blockIdx.x + job.ahead < nmap) {
        // the input rows of the CTA one resident wave on, into L2 (contiguous: its TW rows)
        const BlockWork nb = map[blockIdx.x + job.ahead];
        const SimDev& S2 = sims[nb.sim];
        const long long r0 = (long long)nb.tile * TW;
        const long long nrows = min((long long)TW, (long long)S2.A * S2.B - r0);
        const float* f = field_ptr(S2, job.in_field, nb.comp);
        if (f && nrows > 0)
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(f + r0 * 2 * M),
                         "r"((unsigned)(nrows * 2 * M * sizeof(float))) : "memory");
    }
    const float2* in = reinterpret_cast<const float2*>(field_ptr(S, job.in_field, bw.comp) + (long long)row * (2 * M));
    float2 v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) v[r] = ok ? in[t + T * r] : make_float2(0.f, 0.f);
    FftReg<M, P, false, Lay>::run(v, sh, t, l, S.plan_row.twn);
    // the split needs Z[M - k], held by another thread of the row
#pragma unroll
    for (int m = 0; m < R1; ++m) sh[Lay::at(t + T * m, l)] = v[m];
    __syncthreads();
    if (!ok) return;
    float2* out = S.spec[job.spec_out + bw.comp] + (long long)row * S.Cp;
    const float2* __restrict__ tw = S.row_tw;
#pragma unroll
    for (int m = 0; m < R1; ++m) {
        const int k = t + T * m;
        out[k] = r2c_bin(v[m], sh[Lay::at(k == 0 ? 0 : M - k, l)], __ldg(tw + k));
    }
    if (t == 0) out[M] = r2c_bin(v[0], v[0], __ldg(tw + M));
}

// ---------------------------------------------------------------------------------------------
// C2R + epilogue
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ float2 ld_state(const float* p, long long e) { return *reinterpret_cast<const float2*>(p + e); }
__device__ __forceinline__ void st_state(float* p, long long e, float2 v) { *reinterpret_cast<float2*>(p + e) = v; }
__device__ __forceinline__ float2 ld_medium(const FieldOrScalar& f, long long e) {
    return f.ptr ? __ldg(reinterpret_cast<const float2*>(f.ptr + e)) : make_float2(f.s, f.s);
}
__device__ __forceinline__ float& half(float2& v, int h) { return h ? v.y : v.x; }
__device__ __forceinline__ float2 ld_ro(const float* p, long long e) { return __ldg(reinterpret_cast<const float2*>(p + e)); }

// VAR: launch-shape variants of the same arithmetic (bit 0 halves the pairs whose inputs are loaded
// together, bit 1 swaps two and three CTAs per SM). FWD (velocity and density epilogues): the
// epilogue's output rows are transformed forward again in the same CTA and written as the next
// job's input spectra (job.fwd_spec): the new u_a for the density job; rho0 div u and rho_sum for
// the power-law absorption job, whose rho0 div u field is then not stored at all.
template <int M, int EPI, bool TAPE = false, int VAR = 0, bool FWD = false>
__global__ void __launch_bounds__(256, rowr_minb<M, EPI, TAPE, VAR>()) k_rowr_c2r(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                                  const BlockWork* __restrict__ map, int nmap, RowC2RJob job) {
    pdl_enter();
    using P = RegPlan<M, c2r_r1(M)>;
    using Lay = RowLayout<P, M>;
    constexpr int R1 = P::R1, T = P::T, TW = P::LINES;
    // pairs whose inputs are loaded together (the density update reads the most fields)
    constexpr bool DEN = EPI == EPI_DEN || EPI == EPI_DEN_SRC;
    constexpr bool AEOS = EPI == EPI_ADJ_EOS || EPI == EPI_ADJ_EOS_RHO;
    constexpr int MB0 = (EPI == EPI_DEN_SRC && M <= 128) ? 1 : ((DEN || AEOS || R1 < 4) ? 2 : 4);
    constexpr int MB = (VAR & 1) ? (MB0 > 1 ? MB0 / 2 : 1) : MB0;
    __shared__ float2 sh[Lay::SLOTS];
    extern __shared__ __align__(16) float2 parked[];   // coupled epilogues: [ncomp - 1][R1][256]
    if (blockIdx.x >= nmap) return;
    const BlockWork bw = map[blockIdx.x];
    const SimDev& S = sims[bw.sim];
    if (!gate_open(S, job.gate, bw.comp, *d_t)) return;
    const int t = threadIdx.x % T, l = threadIdx.x / T;
    const int row = bw.tile * TW + l;
    const bool ok = row < S.A * S.B;
    const int comp0 = job.ncomp == 1 ? bw.comp : 0;
    const int ncomp = (EPI == EPI_EOS_ABS && S.absorb != 3) ? 1 : job.ncomp;
    const float2* __restrict__ tw = S.row_tw;
    // The epilogue's field rows of this CTA are contiguous (TW rows of 2M floats): one thread asks
    // for each of them to be brought into L2 now (cp.async.bulk.prefetch), so the epilogue's loads
    // after the inverse transforms find them there. No registers or shared memory are involved.
    if (job.prefetch && threadIdx.x == 0) {
        const long long r0 = (long long)bw.tile * TW;
        const long long nrows = min((long long)TW, (long long)S.A * S.B - r0);
        const unsigned bytes = (unsigned)(nrows * 2 * M * sizeof(float));
        auto pf = [&](const float* f) {
            if (f) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(f + r0 * 2 * M), "r"(bytes) : "memory");
        };
        auto pf64 = [&](const double* f) {   // FP64 accumulators
            if (f) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(f + r0 * 2 * M), "r"(2 * bytes) : "memory");
        };
        // the spectrum rows of the CTA one resident wave on (all its components)
        if (job.ahead > 0 && blockIdx.x + job.ahead < nmap) {
            const BlockWork nb = map[blockIdx.x + job.ahead];
            const SimDev& S2 = sims[nb.sim];
            const long long q0 = (long long)nb.tile * TW;
            const long long nq = min((long long)TW, (long long)S2.A * S2.B - q0);
            const int c0n = job.ncomp == 1 ? nb.comp : 0;
            for (int cc = 0; cc < job.ncomp && nq > 0; ++cc)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(S2.spec[job.spec_in + c0n + cc] + q0 * S2.Cp),
                             "r"((unsigned)(nq * S2.Cp * sizeof(float2))) : "memory");
        }
        // the coupled components after the first are transformed after it: their spectrum rows too
        for (int cc = 1; cc < ncomp; ++cc) {
            const float2* X0 = S.spec[job.spec_in + comp0 + cc] + r0 * S.Cp;
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(X0), "r"((unsigned)(nrows * S.Cp * sizeof(float2)))
                         : "memory");
        }
        if constexpr (EPI == EPI_VEL) {
            pf(S.u[comp0]);
            pf(S.dtor[comp0].ptr);
        } else if constexpr (EPI == EPI_DEN || EPI == EPI_DEN_SRC) {
            for (int a = 0; a < S.dim; ++a) pf(S.rho[a]);
            pf(S.rho0.ptr);
            if (EPI == EPI_DEN_SRC && psrc_gain(S, *d_t) != 0.f) pf(S.psrc_q);
            if (S.eos_pointwise) { pf(S.c2.ptr); if (S.absorb == 1) pf(S.tau.ptr); if (S.nonlinear) pf(S.bona.ptr); }
        } else if constexpr (EPI == EPI_EOS_ABS) {
            pf(S.rho_sum);
            pf(S.c2.ptr);
            pf(S.tau.ptr);
            if (S.absorb == 3) pf(S.eta.ptr);
            if (S.nonlinear) { pf(S.bona.ptr); pf(S.rho0.ptr); }
        } else if constexpr (EPI == EPI_ADJ_VEL || EPI == EPI_ADJ_VEL_RHO) {
            pf(S.adj[ADJ_LU + comp0]);
            pf(S.dtor[comp0].ptr);
            if (EPI == EPI_ADJ_VEL_RHO) { pf(S.adj[ADJ_GP + comp0]); pf64(S.adj_gdtor[comp0]); }
        } else if constexpr (EPI == EPI_ADJ_SUM) {
            if (S.absorb >= 2) { pf(S.c2.ptr); pf(S.tau.ptr); if (S.absorb == 3) pf(S.eta.ptr); }
        } else if constexpr (AEOS) {
            pf(S.adj[ADJ_LP]); pf(S.adj[ADJ_PTP]); pf(S.adj[ADJ_STP]);
            pf(S.c2.ptr); pf(S.rho0.ptr); pf(S.tau.ptr);
            if (S.absorb == 3) { pf(S.eta.ptr); pf(S.adj[ADJ_Q2]); }
            if (S.nonlinear) { pf(S.bona.ptr); pf(S.adj[ADJ_SPRP]); }
            for (int a = 0; a < S.dim; ++a) {
                pf(S.adj[ADJ_LR + a]);
                if (S.nonlinear || EPI == EPI_ADJ_EOS_RHO) pf(S.adj[ADJ_DDP + a]);
            }
            pf64(S.adj_gc);
            if (EPI == EPI_ADJ_EOS_RHO) pf64(S.adj_gr);
        }
    }

    // Z'[k] = (X[k] + conj X[M-k]) + i exp(+2 pi i k / C) (X[k] - conj X[M-k]), X[0] and X[M] real
    float2 v[R1];
    for (int cc = 0; cc < ncomp; ++cc) {
        const float2* X = S.spec[job.spec_in + comp0 + cc] + (long long)row * S.Cp;
#pragma unroll
        for (int m = 0; m < R1; ++m) {
            const int k = t + T * m;
            float2 a0 = make_float2(0.f, 0.f), b0 = a0;
            if (ok) { a0 = X[k]; b0 = X[M - k]; }
            if (k == 0) { a0.y = 0.f; b0.y = 0.f; }
            const float2 s = make_float2(a0.x + b0.x, a0.y - b0.y);
            const float2 dd = make_float2(a0.x - b0.x, a0.y + b0.y);
            const float2 e = cmulc(dd, __ldg(tw + k));
            v[m] = make_float2(s.x - e.y, s.y + e.x);
        }
        FftReg<M, P, true, Lay>::run(v, sh, t, l, S.plan_row.twn);
        if (cc + 1 < ncomp) {
#pragma unroll
            for (int m = 0; m < R1; ++m) parked[(cc * R1 + m) * 256 + threadIdx.x] = v[m];
        }
    }
    // FWD: the forward R2C of the epilogue's outputs (v; the density epilogue's rho_sum in parked
    // slot 0); the number of transforms is uniform over the CTA (one simulation per CTA)
    auto forward_tail = [&]() {
        if constexpr (FWD) {
            constexpr bool PER_COMP = EPI == EPI_VEL || EPI == EPI_ADJ_VEL || EPI == EPI_ADJ_VEL_RHO;
            static_assert(PER_COMP || EPI == EPI_DEN || EPI == EPI_DEN_SRC, "row fusion");
            const int nf = PER_COMP ? 1 : (S.absorb == 3 ? 2 : (S.absorb == 2 ? 1 : 0));
            for (int f = 0; f < nf; ++f) {
                if (f == 1) {
#pragma unroll
                    for (int m = 0; m < R1; ++m) v[m] = parked[m * 256 + threadIdx.x];
                }
                const int o = PER_COMP ? comp0 : f;
                rowr_forward<M, P, Lay>(v, sh, t, l, S.plan_row.twn, tw, S.spec[job.fwd_spec + o] + (long long)row * S.Cp, ok);
            }
        }
    };
    // rows past the end skip the epilogue; with FWD they still take part in the forward transforms'
    // barriers, which every thread reaches at the same instruction (one call below)
    if constexpr (!FWD) {
        if (!ok) return;
    }
    if (ok) {
        const long long rbase = (long long)row * (2 * M);
        const int ca = row / S.B, cb = row - ca * S.B;
        const int D = S.dim;
        // samples 2n, 2n+1 of component cc (pair index m)
        auto dpair = [&](int cc, int m) { return cc + 1 < ncomp ? parked[(cc * R1 + m) * 256 + threadIdx.x] : v[m]; };
        // per-axis profiles: constant along the row except for the row's own axis (a = D - 1), which
        // is read at samples 2n, 2n+1
        auto row_const = [&](const float* vec, int a) { return __ldg(vec + (a + 3 - D == 0 ? ca : cb)); };
        auto row_pair = [&](const float* vec, int n) { return __ldg(reinterpret_cast<const float2*>(vec) + n); };
        // precorrected additive pressure source: rho_a += signal[t] psrc_q / d_a while it lasts
        // (sg_d[a] = signal[t] / d_a; the field is not read, and 0 is added, once the signal has ended)
        const float sgain = EPI == EPI_DEN_SRC ? psrc_gain(S, *d_t) : 0.f;
        float sg_d[kMaxComp];
#pragma unroll
        for (int a = 0; a < kMaxComp; ++a) sg_d[a] = (EPI == EPI_DEN_SRC && a < S.dim) ? sgain * S.ax[a].inv_d : 0.f;

#pragma unroll
        for (int m0 = 0; m0 < R1; m0 += MB) {
            if constexpr (EPI == EPI_STORE) {
                for (int cc = 0; cc < ncomp; ++cc) {
                    float* out = field_ptr(S, job.out_field, comp0 + cc);
#pragma unroll
                    for (int b = 0; b < MB; ++b) st_state(out, rbase + 2 * (t + T * (m0 + b)), dpair(cc, m0 + b));
                }
            } else if constexpr (EPI == EPI_VEL || EPI == EPI_VEL_INIT || EPI == EPI_ADD_U) {
                // u = pml_sg (pml_sg u - dt/rho_sg d)   (KSpaceFirstOrder.swift:453-454)
                // u = (dt/rho_sg / 2) d                 (KSpaceFirstOrder.swift:519-520)
                // u = u + d                             (additive velocity source)
                const int a = comp0;
                float* u = S.u[a];
                const bool along_row = a == D - 1;
                const float sgc = (EPI == EPI_VEL && !along_row) ? row_const(S.ax[a].pml_sg, a) : 0.f;
                float2 uu[MB], dr[MB], sg[MB];
#pragma unroll
                for (int b = 0; b < MB; ++b) {
                    const int n = t + T * (m0 + b);
                    const long long e = rbase + 2 * n;
                    if (EPI != EPI_VEL_INIT) uu[b] = ld_state(u, e);
                    if (EPI != EPI_ADD_U) dr[b] = ld_medium(S.dtor[a], e);
                    if (EPI == EPI_VEL) sg[b] = along_row ? row_pair(S.ax[a].pml_sg, n) : make_float2(sgc, sgc);
                }
#pragma unroll
                for (int b = 0; b < MB; ++b) {
                    const float2 d = v[m0 + b];
                    float2 o;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const float dh = h ? d.y : d.x;
                        if (EPI == EPI_VEL) half(o, h) = half(sg[b], h) * (half(sg[b], h) * half(uu[b], h) - half(dr[b], h) * dh);
                        else if (EPI == EPI_VEL_INIT) half(o, h) = (half(dr[b], h) / 2.f) * dh;
                        else half(o, h) = half(uu[b], h) + dh;
                    }
                    st_state(u, rbase + 2 * (t + T * (m0 + b)), o);
                    if constexpr (FWD) v[m0 + b] = o;
                }
            } else if constexpr (DEN || EPI == EPI_ADD_RHO) {
                // density (KSpaceFirstOrder.swift:457-465) or additive pressure source
                // (KSpaceFirstOrder.swift:167-172), then the pointwise equation of state when there is one
                float2 ro[kMaxComp][MB], pmr[MB], r0[MB], c2[MB], tau[MB], bona[MB], eta[MB], sq[MB];
                float pmc[kMaxComp - 1];
#pragma unroll
                for (int a = 0; a < kMaxComp - 1; ++a)
                    if (DEN && a < D - 1) pmc[a] = row_const(S.ax[a].pml, a);
                const bool need_r0 = DEN || S.nonlinear;
#pragma unroll
                for (int b = 0; b < MB; ++b) {
                    const int n = t + T * (m0 + b);
                    const long long e = rbase + 2 * n;
#pragma unroll
                    for (int a = 0; a < kMaxComp; ++a)
                        if (a < D) ro[a][b] = ld_state(S.rho[a], e);
                    if (DEN) pmr[b] = row_pair(S.ax[D - 1].pml, n);
                    if (EPI == EPI_DEN_SRC) sq[b] = sgain != 0.f ? ld_ro(S.psrc_q, e) : make_float2(0.f, 0.f);
                    if (need_r0) r0[b] = ld_medium(S.rho0, e);
                    if (S.eos_pointwise) {
                        c2[b] = ld_medium(S.c2, e);
                        if (S.absorb == 1) tau[b] = ld_medium(S.tau, e);
                        if (S.nonlinear) bona[b] = ld_medium(S.bona, e);
                        if (EPI == EPI_ADD_RHO && S.absorb == 1) eta[b] = ld_state(S.div_term, e);
                    }
                }
#pragma unroll
                for (int b = 0; b < MB; ++b) {
                    const int m = m0 + b;
                    const long long e = rbase + 2 * (t + T * m);
                    float2 rn[kMaxComp], rs2, dv2, p2;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const float r0v = need_r0 ? half(r0[b], h) : 0.f;
                        float rs = 0.f, divterm = 0.f;
                        if (DEN) {
                            float nl = 1.f;
                            if (S.nonlinear) {
                                float rp = 0.f;
#pragma unroll
                                for (int a = 0; a < kMaxComp; ++a)
                                    if (a < D) rp = a == 0 ? half(ro[a][b], h) : rp + half(ro[a][b], h);
                                nl = (2.f * rp + r0v) / r0v;
                            }
                            const float dtr = S.dt * r0v;   // dt * rho0 in FP32 (KSpaceFirstOrder.swift:400)
                            float dv = 0.f;
#pragma unroll
                            for (int a = 0; a < kMaxComp; ++a)
                                if (a < D) {
                                    float2 dp = dpair(a, m);
                                    const float d = half(dp, h);
                                    const float pmv = a == D - 1 ? half(pmr[b], h) : pmc[a < kMaxComp - 1 ? a : 0];
                                    const float mass = S.nonlinear ? dtr * d * nl : dtr * d;
                                    float r = pmv * (pmv * half(ro[a][b], h) - mass);
                                    if (EPI == EPI_DEN_SRC) r = r + sg_d[a] * half(sq[b], h);
                                    half(rn[a], h) = r;
                                    rs = a == 0 ? r : rs + r;
                                    dv = a == 0 ? d : dv + d;
                                }
                            if (S.absorb >= 1) divterm = r0v * dv;
                        } else {
                            const float d = h ? v[m].y : v[m].x;
#pragma unroll
                            for (int a = 0; a < kMaxComp; ++a)
                                if (a < D) {
                                    const float r = half(ro[a][b], h) + d * S.ax[a].inv_d;
                                    half(rn[a], h) = r;
                                    rs = a == 0 ? r : rs + r;
                                }
                            if (S.absorb == 1) divterm = half(eta[b], h);
                        }
                        half(rs2, h) = rs;
                        half(dv2, h) = divterm;
                        if (S.eos_pointwise) {   // p = c0^2 (rho + tau divterm + B/A rho^2 / (2 rho0))
                            float ee = rs;
                            if (S.absorb == 1) ee = ee + half(tau[b], h) * divterm;
                            if (S.nonlinear) ee = ee + half(bona[b], h) * (rs * rs) / (2.f * r0v);
                            half(p2, h) = half(c2[b], h) * ee;
                        }
                    }
#pragma unroll
                    for (int a = 0; a < kMaxComp; ++a)
                        if (a < D) st_state(S.rho[a], e, rn[a]);
                    st_state(S.rho_sum, e, rs2);
                    if constexpr (FWD) {   // every input of pair m is consumed: its slots take the outputs
                        v[m] = dv2;
                        parked[m * 256 + threadIdx.x] = rs2;
                    }
                    if (DEN && S.absorb >= 1 && !(FWD && S.absorb >= 2)) st_state(S.div_term, e, dv2);
                    if (S.eos_pointwise) st_state(S.p, e, p2);
                    if constexpr (TAPE) {   // the adjoint's recompute: d_a = D-_a u_a, and S, p, div when they are final here
                        const AdjTapeEntry& te = S.tape[*d_t];
                        if (DEN && (S.nonlinear || S.adj_gr)) {   // B/A, or the density gradient
#pragma unroll
                            for (int a = 0; a < kMaxComp; ++a)
                                if (a < D) st_state(te.dd[a], e, dpair(a, m));
                        }
                        if (S.eos_pointwise) {
                            st_state(te.s, e, rs2);
                            st_state(te.p, e, p2);
                        }
                        if (DEN && S.absorb == 1) st_state(te.div, e, dv2);
                    }
                }
            } else if constexpr (EPI == EPI_ADJ_VEL || EPI == EPI_ADJ_VEL_RHO) {
                // adjoint of the velocity update (kw_adjoint.cu)
                const int a = comp0;
                float* lu = S.adj[ADJ_LU + a];
                float* w = S.adj[ADJ_W + a];
                const bool along_row = a == D - 1;
                const float sgc = along_row ? 0.f : row_const(S.ax[a].pml_sg, a);
                float2 uu[MB], dr[MB], sg[MB];
#pragma unroll
                for (int b = 0; b < MB; ++b) {
                    const int n = t + T * (m0 + b);
                    const long long e = rbase + 2 * n;
                    uu[b] = ld_state(lu, e);
                    dr[b] = ld_medium(S.dtor[a], e);
                    sg[b] = along_row ? row_pair(S.ax[a].pml_sg, n) : make_float2(sgc, sgc);
                }
#pragma unroll
                for (int b = 0; b < MB; ++b) {
                    const float2 d = v[m0 + b];
                    float2 lo, wo;
                    const long long e = rbase + 2 * (t + T * (m0 + b));
                    if constexpr (EPI == EPI_ADJ_VEL_RHO) {   // dL/d dtor_a += -sg_a g_a mu_a, g_a = D+_a p(t-1)
                        const float2 gp = ld_ro(S.adj[ADJ_GP + a], e);
                        double2 gd = *reinterpret_cast<const double2*>(S.adj_gdtor[a] + e);
                        gd.x -= (double)sg[b].x * gp.x * (uu[b].x - d.x);
                        gd.y -= (double)sg[b].y * gp.y * (uu[b].y - d.y);
                        *reinterpret_cast<double2*>(S.adj_gdtor[a] + e) = gd;
                    }
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const float mu = half(uu[b], h) - (h ? d.y : d.x);
                        half(lo, h) = half(sg[b], h) * half(sg[b], h) * mu;
                        half(wo, h) = half(sg[b], h) * half(dr[b], h) * mu;
                    }
                    st_state(lu, e, lo);
                    st_state(w, e, wo);
                    if constexpr (FWD) v[m0 + b] = wo;
                }
            } else if constexpr (EPI == EPI_ADJ_SUM) {
                // lambda_p = sum_a d_a and the next reverse step's absorption inputs (the medium of the
                // MB pairs is loaded before the first store, which the compiler may not reorder)
                float2 c2[MB], tau[MB], eta[MB];
                if (S.absorb >= 2) {
#pragma unroll
                    for (int b = 0; b < MB; ++b) {
                        const long long e = rbase + 2 * (t + T * (m0 + b));
                        c2[b] = ld_medium(S.c2, e);
                        tau[b] = ld_medium(S.tau, e);
                        if (S.absorb == 3) eta[b] = ld_medium(S.eta, e);
                    }
                }
#pragma unroll
                for (int b = 0; b < MB; ++b) {
                    const int m = m0 + b;
                    const long long e = rbase + 2 * (t + T * m);
                    float2 s2 = dpair(0, m);
                    for (int cc = 1; cc < ncomp; ++cc) {
                        const float2 dp = dpair(cc, m);
                        s2.x += dp.x;
                        s2.y += dp.y;
                    }
                    st_state(S.adj[ADJ_LP], e, s2);
                    if (S.absorb >= 2) {
                        st_state(S.adj[ADJ_X1], e, make_float2(tau[b].x * c2[b].x * s2.x, tau[b].y * c2[b].y * s2.y));
                        if (S.absorb == 3)
                            st_state(S.adj[ADJ_X2], e, make_float2(eta[b].x * c2[b].x * s2.x, eta[b].y * c2[b].y * s2.y));
                    }
                }
            } else if constexpr (AEOS) {
                // the reverse equation of state of kw_adjoint.cu (k_adj_eos), with the absorption
                // filters' outputs d = A1(tau c^2 lambda_p), A2(eta c^2 lambda_p), A2(S(t)) in hand
                const int tt = *d_t;
                const bool src_on = S.has_p && S.psrc.mode == 1 && tt < S.psrc.len;   // additive source active
                if (m0 == 0 && blockIdx.x == 0 && threadIdx.x == 0) *S.adj_rev -= 1;
                float pmc[kMaxComp - 1];
#pragma unroll
                for (int a = 0; a < kMaxComp - 1; ++a)
                    if (a < D - 1) pmc[a] = row_const(S.ax[a].pml, a);
#pragma unroll
                for (int b = 0; b < MB; ++b) {
                    const int m = m0 + b;
                    const int n = t + T * m;
                    const long long e = rbase + 2 * n;
                    // lambda_p and the tape are read-only here: loaded through the non-coherent path, so
                    // the compiler may issue them ahead of the previous pair's stores
                    const float2 lp = ld_ro(S.adj[ADJ_LP], e), pv = ld_ro(S.adj[ADJ_PTP], e), sv = ld_ro(S.adj[ADJ_STP], e);
                    const float2 c2 = ld_medium(S.c2, e), r0 = ld_medium(S.rho0, e), tau = ld_medium(S.tau, e);
                    float2 eta = make_float2(0.f, 0.f), bona = eta, spv = eta;
                    if (S.absorb == 3) eta = ld_medium(S.eta, e);
                    if (S.nonlinear) { bona = ld_medium(S.bona, e); spv = ld_ro(S.adj[ADJ_SPRP], e); }
                    float2 lr[kMaxComp], dd[kMaxComp];
#pragma unroll
                    for (int a = 0; a < kMaxComp; ++a)
                        if (a < D) {
                            lr[a] = ld_state(S.adj[ADJ_LR + a], e);
                            if (S.nonlinear || EPI == EPI_ADJ_EOS_RHO) dd[a] = ld_ro(S.adj[ADJ_DDP + a], e);
                        }
                    double2 grv = make_double2(0.0, 0.0);
                    if constexpr (EPI == EPI_ADJ_EOS_RHO) grv = *reinterpret_cast<const double2*>(S.adj_gr + e);
                    const float2 pmr = row_pair(S.ax[D - 1].pml, n);
                    const float2 a1 = dpair(0, m);
                    float2 a2 = make_float2(0.f, 0.f), q2 = a2;
                    if (S.absorb == 3) { a2 = dpair(1, m); q2 = ld_ro(S.adj[ADJ_Q2], e); }
                    double2 gcv = *reinterpret_cast<const double2*>(S.adj_gc + e);
                    float2 lro[kMaxComp], wo[kMaxComp], sg2;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const float cc2 = h ? c2.y : c2.x, c = sqrtf(cc2);
                        const float lpv = h ? lp.y : lp.x, p_ = h ? pv.y : pv.x, s_ = h ? sv.y : sv.x;
                        const float rr0 = h ? r0.y : r0.x, ta = h ? tau.y : tau.x, et = h ? eta.y : eta.x;
                        const float bo = h ? bona.y : bona.x;
                        double E = (double)p_ / cc2 - s_;
                        if (S.nonlinear) E -= (double)bo * s_ * s_ / (2.0 * rr0);
                        double term = (double)(S.adj_y - 1.f) * E;
                        if (S.absorb == 3) term -= (double)et * (h ? q2.y : q2.x);
                        const double dpdc = 2.0 * (double)p_ / c + (double)c * term;
                        if (h) gcv.y += (double)lpv * dpdc; else gcv.x += (double)lpv * dpdc;
                        const float lE = cc2 * lpv;
                        float lS = lE;
                        if (S.nonlinear) lS += lE * bo * s_ / rr0;
                        if (S.absorb == 3) lS -= h ? a2.y : a2.x;
                        const float ldiv = h ? a1.y : a1.x;
                        const float nl = S.nonlinear ? (2.f * (h ? spv.y : spv.x) + rr0) / rr0 : 1.f;
                        const float dtr = S.dt * rr0;
                        float lam[kMaxComp], pmv[kMaxComp];
                        float lsprev = 0.f, sig = 0.f;
#pragma unroll
                        for (int a = 0; a < kMaxComp; ++a) {
                            if (a >= D) break;
                            pmv[a] = a == D - 1 ? (h ? pmr.y : pmr.x) : pmc[a < kMaxComp - 1 ? a : 0];
                            lam[a] = (h ? lr[a].y : lr[a].x) + lS;
                            half(wo[a], h) = rr0 * ldiv - pmv[a] * dtr * nl * lam[a];
                            if (S.nonlinear) lsprev += -2.f * S.dt * pmv[a] * (h ? dd[a].y : dd[a].x) * lam[a];
                            sig += lam[a] * S.ax[a].inv_d;
                        }
#pragma unroll
                        for (int a = 0; a < kMaxComp; ++a) {
                            if (a >= D) break;
                            half(lro[a], h) = pmv[a] * pmv[a] * lam[a] + lsprev;
                        }
                        half(sg2, h) = sig;
                        if constexpr (EPI == EPI_ADJ_EOS_RHO) {
                            // direct terms of dL/drho0: the absorption input rho0 div, B/A S^2 / (2 rho0),
                            // and d(dt rho0 nl) / d rho0 = dt in each density update
                            float sd = 0.f;
                            double g = 0.0;
#pragma unroll
                            for (int a = 0; a < kMaxComp; ++a) {
                                if (a >= D) break;
                                const float dv = h ? dd[a].y : dd[a].x;
                                sd += dv;
                                g -= (double)pmv[a] * S.dt * dv * lam[a];
                            }
                            g += (double)ldiv * sd;
                            if (S.nonlinear) g -= (double)lE * bo * s_ * s_ / (2.0 * (double)rr0 * rr0);
                            if (h) grv.y += g; else grv.x += g;
                        }
                    }
                    *reinterpret_cast<double2*>(S.adj_gc + e) = gcv;
                    if constexpr (EPI == EPI_ADJ_EOS_RHO) *reinterpret_cast<double2*>(S.adj_gr + e) = grv;
#pragma unroll
                    for (int a = 0; a < kMaxComp; ++a)
                        if (a < D) { st_state(S.adj[ADJ_LR + a], e, lro[a]); st_state(S.adj[ADJ_W + a], e, wo[a]); }
                    if (src_on) st_state(S.adj[ADJ_SIG], e, sg2);
                }
            } else if constexpr (EPI == EPI_EOS_ABS) {
                // power-law absorption / dispersion (KSpaceFirstOrder.swift:836-845)
                float2 rs[MB], c2[MB], tau[MB], eta[MB], bona[MB], r0[MB];
#pragma unroll
                for (int b = 0; b < MB; ++b) {
                    const long long e = rbase + 2 * (t + T * (m0 + b));
                    rs[b] = ld_ro(S.rho_sum, e);   // read-only here: may be issued ahead of the stores
                    c2[b] = ld_medium(S.c2, e);
                    tau[b] = ld_medium(S.tau, e);
                    if (S.absorb == 3) eta[b] = ld_medium(S.eta, e);
                    if (S.nonlinear) { bona[b] = ld_medium(S.bona, e); r0[b] = ld_medium(S.rho0, e); }
                }
#pragma unroll
                for (int b = 0; b < MB; ++b) {
                    const int m = m0 + b;
                    const float2 d0 = dpair(0, m);
                    float2 d1 = make_float2(0.f, 0.f);
                    if (S.absorb == 3) d1 = dpair(1, m);
                    float2 p2;
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const float r = half(rs[b], h);
                        float term = half(tau[b], h) * (h ? d0.y : d0.x);
                        if (S.absorb == 3) term = term - half(eta[b], h) * (h ? d1.y : d1.x);
                        float ee = r + term;
                        if (S.nonlinear) ee = ee + half(bona[b], h) * (r * r) / (2.f * half(r0[b], h));
                        half(p2, h) = half(c2[b], h) * ee;
                    }
                    st_state(S.p, rbase + 2 * (t + T * m), p2);
                    if constexpr (TAPE) {   // the adjoint's recompute keeps p, S and A2(S)
                        const AdjTapeEntry& te = S.tape[*d_t];
                        const long long e = rbase + 2 * (t + T * m);
                        st_state(te.p, e, p2);
                        st_state(te.s, e, rs[b]);
                        if (S.absorb == 3) st_state(te.q2, e, d1);
                    }
                }
            }
        }
    }
    forward_tail();
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
template <int M>
static size_t rowr_park_bytes(int ncomp) { return (size_t)(ncomp > 1 ? ncomp - 1 : 0) * c2r_r1(M) * 256 * sizeof(float2); }

template <int EPI, bool TAPE = false>
static void set_rowr_attrs(int optin) {
#define KW_SET(m) set_max_smem((const void*)k_rowr_c2r<m, EPI, TAPE>, optin);
    KW_REG_ROW_SIZES(KW_SET)
#undef KW_SET
    if constexpr (!TAPE && (EPI == EPI_DEN || EPI == EPI_DEN_SRC)) {
#define KW_SET(m) set_max_smem((const void*)k_rowr_c2r<m, EPI, false, 0, true>, optin);
        KW_REG_ROW_SIZES(KW_SET)
#undef KW_SET
    }
    set_max_smem((const void*)k_rowr_c2r<128, EPI, TAPE, 1>, optin);
    set_max_smem((const void*)k_rowr_c2r<128, EPI, TAPE, 2>, optin);
    set_max_smem((const void*)k_rowr_c2r<128, EPI, TAPE, 3>, optin);
    if constexpr (!TAPE && (EPI == EPI_DEN || EPI == EPI_DEN_SRC)) {
        set_max_smem((const void*)k_rowr_c2r<128, EPI, false, 1, true>, optin);
        set_max_smem((const void*)k_rowr_c2r<128, EPI, false, 2, true>, optin);
        set_max_smem((const void*)k_rowr_c2r<128, EPI, false, 3, true>, optin);
    }
}

// launch-shape variant of the 128-point C2R epilogues (KW_C2R_VAR = three digits for the density,
// source density and power-law EoS epilogues; default 000)
static int c2r_var(int epi) {
    static int v[3] = {-1, 0, 0};
    if (v[0] < 0) {
        v[0] = v[1] = v[2] = 0;
        if (const char* e = std::getenv("KW_C2R_VAR"))
            for (int i = 0; i < 3 && e[i]; ++i) v[i] = (e[i] - '0') & 3;
    }
    return epi == EPI_DEN ? v[0] : (epi == EPI_DEN_SRC ? v[1] : (epi == EPI_EOS_ABS ? v[2] : 0));
}

template <int M, int EPI, bool FWD = false>
static void launch_var(int var, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap, const RowC2RJob& job,
                       size_t smem, cudaStream_t st) {
    if constexpr (M == 128) {
        if (var == 1) { launch_pdl(k_rowr_c2r<M, EPI, false, 1, FWD>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job); return; }
        if (var == 2) { launch_pdl(k_rowr_c2r<M, EPI, false, 2, FWD>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job); return; }
        if (var == 3) { launch_pdl(k_rowr_c2r<M, EPI, false, 3, FWD>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job); return; }
    }
    launch_pdl(k_rowr_c2r<M, EPI, false, 0, FWD>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job);
}

void init_rowr_attributes(int optin) {
    set_rowr_attrs<EPI_DEN>(optin);
    set_rowr_attrs<EPI_DEN_SRC>(optin);
    set_rowr_attrs<EPI_EOS_ABS>(optin);
    set_rowr_attrs<EPI_DEN, true>(optin);
    set_rowr_attrs<EPI_EOS_ABS, true>(optin);
    set_rowr_attrs<EPI_ADJ_SUM>(optin);
    set_rowr_attrs<EPI_ADJ_EOS>(optin);
    set_rowr_attrs<EPI_ADJ_EOS_RHO>(optin);
}

void launch_rowr_r2c(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                     const RowR2CJob& job, int M) {
    if (nmap <= 0) return;
    switch (M) {
#define KW_CASE(m) \
    case m: launch_pdl(k_rowr_r2c<m>, nmap, 256, 0, st, d_sims, d_t, map, nmap, job); break;
        KW_REG_ROW_SIZES(KW_CASE)
#undef KW_CASE
        default: break;
    }
}

template <int M>
static void launch_c2r_m(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                         const RowC2RJob& job) {
    const size_t smem = rowr_park_bytes<M>(job.ncomp);
    switch (job.epi) {
        case EPI_STORE: launch_pdl(k_rowr_c2r<M, EPI_STORE>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job); break;
        case EPI_VEL:
            if (job.fwd) launch_pdl(k_rowr_c2r<M, EPI_VEL, false, 0, true>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job);
            else launch_pdl(k_rowr_c2r<M, EPI_VEL>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job);
            break;
        case EPI_VEL_INIT: launch_pdl(k_rowr_c2r<M, EPI_VEL_INIT>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job); break;
        case EPI_ADD_U: launch_pdl(k_rowr_c2r<M, EPI_ADD_U>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job); break;
        case EPI_DEN:
            if (job.tape) launch_pdl(k_rowr_c2r<M, EPI_DEN, true>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job);
            else if (job.fwd) launch_var<M, EPI_DEN, true>(c2r_var(EPI_DEN), d_sims, d_t, map, nmap, job, smem, st);
            else launch_var<M, EPI_DEN>(c2r_var(EPI_DEN), d_sims, d_t, map, nmap, job, smem, st);
            break;
        case EPI_DEN_SRC:
            if (job.fwd) launch_var<M, EPI_DEN_SRC, true>(c2r_var(EPI_DEN_SRC), d_sims, d_t, map, nmap, job, smem, st);
            else launch_var<M, EPI_DEN_SRC>(c2r_var(EPI_DEN_SRC), d_sims, d_t, map, nmap, job, smem, st);
            break;
        case EPI_ADD_RHO:
            if (job.tape) launch_pdl(k_rowr_c2r<M, EPI_ADD_RHO, true>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job);
            else launch_pdl(k_rowr_c2r<M, EPI_ADD_RHO>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job);
            break;
        case EPI_EOS_ABS:
            if (job.tape) launch_pdl(k_rowr_c2r<M, EPI_EOS_ABS, true>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job);
            else launch_var<M, EPI_EOS_ABS>(c2r_var(EPI_EOS_ABS), d_sims, d_t, map, nmap, job, smem, st);
            break;
        case EPI_ADJ_VEL:
            if (job.fwd) launch_pdl(k_rowr_c2r<M, EPI_ADJ_VEL, false, 0, true>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job);
            else launch_pdl(k_rowr_c2r<M, EPI_ADJ_VEL>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job);
            break;
        case EPI_ADJ_VEL_RHO:
            if (job.fwd) launch_pdl(k_rowr_c2r<M, EPI_ADJ_VEL_RHO, false, 0, true>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job);
            else launch_pdl(k_rowr_c2r<M, EPI_ADJ_VEL_RHO>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job);
            break;
        case EPI_ADJ_SUM: launch_pdl(k_rowr_c2r<M, EPI_ADJ_SUM>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job); break;
        case EPI_ADJ_EOS: launch_pdl(k_rowr_c2r<M, EPI_ADJ_EOS>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job); break;
        case EPI_ADJ_EOS_RHO: launch_pdl(k_rowr_c2r<M, EPI_ADJ_EOS_RHO>, nmap, 256, smem, st, d_sims, d_t, map, nmap, job); break;
        default: break;
    }
}

void launch_rowr_c2r(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                     const RowC2RJob& job, int M) {
    if (nmap <= 0) return;
    switch (M) {
#define KW_CASE(m) \
    case m: launch_c2r_m<m>(st, d_sims, d_t, map, nmap, job); break;
        KW_REG_ROW_SIZES(KW_CASE)
#undef KW_CASE
        default: break;
    }
}

}  // namespace kw
