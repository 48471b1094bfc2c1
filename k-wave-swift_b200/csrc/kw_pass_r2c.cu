// kw_pass_r2c.cu — row pass R2C: real rows (contiguous axis C) -> half-spectrum rows.
#include "kw_pass_common.cuh"

namespace kw {

__device__ __forceinline__ void r2c_prefetch(const SimDev& G, const BlockWork bw, const RowR2CJob& job, float2* buf, int t) {
    if (!gate_open(G, job.gate, bw.comp, t)) return;
    const int C = G.C, rows = G.A * G.B;
    const bool odd = (C & 1) != 0;
    const int M = odd ? C : C / 2;
    const int L = row_lines(M);
    const int LDI = L + 1;
    const int r0 = bw.tile * L;
    const int nl = min(L, rows - r0);
    const float* in = field_ptr(G, job.in_field, bw.comp) + (long long)r0 * C;
    for (int w = threadIdx.x; w < nl * M; w += blockDim.x) {
        const int l = w / M, m = w - l * M;
        float2* d = buf + m * LDI + l;
        if (!odd) {
            cp_async8(d, in + (long long)l * C + 2 * m);
        } else {
            cp_async4(d, in + (long long)l * C + m);
            d->y = 0.f;
        }
    }
}

template <int MT>
__device__ __forceinline__ void r2c_compute(const SimDev& S, const BlockWork bw, const RowR2CJob& job, float2* buf,
                                            float2* tmp) {
    constexpr bool FIX = MT > 0;
    constexpr int LT = FIX ? row_lines(MT) : 1;
    const int C = S.C, rows = S.A * S.B;
    const bool odd = !FIX && (C & 1) != 0;
    const int M = FIX ? MT : (odd ? C : C / 2);
    const int L = FIX ? LT : row_lines(M);
    const int LDI = L + 1;
    const int r0 = bw.tile * L;
    const int nl = min(L, rows - r0);
    const float2* Z;
    if constexpr (FIX) Z = fft_tile<MT, LT, LT + 1, false>(buf, tmp, S.plan_row.twn, nl);
    else Z = fft_lines<false>(buf, tmp, S.plan_row, nl, 1, LDI, true);

    float2* out = S.spec[job.spec_out + bw.comp] + (long long)r0 * S.Cp;
    const int Ch = S.Ch;
    const OpSpec op = job.op[bw.comp];
    for (int w = threadIdx.x; w < nl * Ch; w += blockDim.x) {
        const int l = w / Ch, k = w - l * Ch;
        float2 X;
        if (!odd) {
            const float2 zk = Z[(k == M ? 0 : k) * LDI + l];
            const float2 zm = Z[(k == 0 ? 0 : M - k) * LDI + l];
            const float2 E = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
            const float2 D = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y + zm.y));
            const float2 O = make_float2(D.y, -D.x);  // -i D
            X = cadd(E, cmul(O, __ldg(S.row_tw + k)));
        } else {
            X = Z[k * LDI + l];
        }
        if (job.apply_op) X = cmul(X, op_factor(S, op, 0, 0, k, (long long)(r0 + l) * S.Cp + k));
        out[(long long)l * S.Cp + k] = X;
    }
}

template <int MT>
__global__ void __launch_bounds__(256) k_row_r2c(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                                 const BlockWork* __restrict__ map, int nmap, RowR2CJob job) {
    extern __shared__ __align__(16) float2 sm[];
    __shared__ SimDev S;
    int cur = -1;
    const int t = *d_t;
    const long long te = job.tile_elems;
    float2* tmp = sm + 2 * te;
    int idx = blockIdx.x;
    if (idx < nmap) { const BlockWork b = map[idx]; r2c_prefetch(sims[b.sim], b, job, sm, t); }
    cp_commit();
#pragma unroll 1
    for (int k = 0; idx < nmap; ++k, idx += gridDim.x) {
        const int nidx = idx + gridDim.x;
        if (nidx < nmap) { const BlockWork b = map[nidx]; r2c_prefetch(sims[b.sim], b, job, sm + ((k + 1) & 1) * te, t); }
        cp_commit();
        cp_wait<1>();
        const BlockWork bw = map[idx];
        use_sim(S, cur, sims, bw.sim);
        if (gate_open(S, job.gate, bw.comp, t)) r2c_compute<MT>(S, bw, job, sm + (k & 1) * te, tmp);
        __syncthreads();
    }
    cp_wait<0>();
}

void init_r2c_attributes(int optin) {
#define KW_SET(m) set_max_smem((const void*)k_row_r2c<m>, optin);
    KW_FFT_SIZES(KW_SET)
#undef KW_SET
    set_max_smem((const void*)k_row_r2c<0>, optin);
}

void launch_row_r2c(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                    const RowR2CJob& job, size_t smem, int size_class) {
    if (nmap <= 0) return;
    switch (size_class) {
#define KW_CASE(m) \
    case m: k_row_r2c<m><<<persistent_grid((const void*)k_row_r2c<m>, smem, nmap), 256, smem, st>>>(d_sims, d_t, map, nmap, job); break;
        KW_FFT_SIZES(KW_CASE)
#undef KW_CASE
        default:
            k_row_r2c<0><<<persistent_grid((const void*)k_row_r2c<0>, smem, nmap), 256, smem, st>>>(d_sims, d_t, map, nmap, job);
            break;
    }
}

}  // namespace kw
