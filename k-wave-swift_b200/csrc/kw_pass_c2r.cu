// kw_pass_c2r.cu — row pass C2R of half-spectrum rows with the physics update as the epilogue.
#include "kw_pass_common.cuh"

namespace kw {

// Fields an epilogue reads, staged row by row next to the spectrum rows.
enum AuxSlot { AX_F0 = 0, AX_F1, AX_F2, AX_RHO0, AX_C2, AX_TAU, AX_BONA, AX_ETA, AX_COUNT };

struct AuxPlan {
    const float* src[AX_COUNT];
    int8_t slot[AX_COUNT];   // compacted position of each field, -1 when not staged
    int n;
};

__device__ __forceinline__ AuxPlan aux_plan(const SimDev& S, const RowC2RJob& job, int comp0) {
    AuxPlan a;
    for (int i = 0; i < AX_COUNT; ++i) { a.src[i] = nullptr; a.slot[i] = -1; }
    switch (job.epi) {
        case EPI_VEL: a.src[AX_F0] = S.u[comp0]; a.src[AX_F1] = S.dtor[comp0].ptr; break;
        case EPI_VEL_INIT: a.src[AX_F1] = S.dtor[comp0].ptr; break;
        case EPI_ADD_U: a.src[AX_F0] = S.u[comp0]; break;
        case EPI_DEN:
        case EPI_DEN_SRC:
        case EPI_ADD_RHO:
            for (int d = 0; d < S.dim; ++d) a.src[AX_F0 + d] = S.rho[d];
            if (S.nonlinear || S.absorb >= 1 || job.epi != EPI_ADD_RHO) a.src[AX_RHO0] = S.rho0.ptr;
            if (S.eos_pointwise) {
                a.src[AX_C2] = S.c2.ptr;
                if (S.absorb == 1) a.src[AX_TAU] = S.tau.ptr;
                if (S.nonlinear) a.src[AX_BONA] = S.bona.ptr;
                if (job.epi == EPI_ADD_RHO && S.absorb == 1) a.src[AX_ETA] = S.div_term;  // Stokes term input
            }
            break;
        case EPI_EOS_ABS:
            a.src[AX_F0] = S.rho_sum;
            a.src[AX_C2] = S.c2.ptr;
            a.src[AX_TAU] = S.tau.ptr;
            if (S.absorb == 3) a.src[AX_ETA] = S.eta.ptr;
            if (S.nonlinear) { a.src[AX_BONA] = S.bona.ptr; a.src[AX_RHO0] = S.rho0.ptr; }
            break;
        default: break;
    }
    a.n = 0;
    for (int i = 0; i < AX_COUNT; ++i)
        if (a.src[i]) a.slot[i] = (int8_t)a.n++;
    return a;
}

struct RowTile {
    int M, L, RPC, r0, nl, ncomp, comp0;
    bool odd;
};

__device__ __forceinline__ RowTile c2r_tile(const SimDev& G, const RowC2RJob& job, const BlockWork bw) {
    RowTile r;
    const int C = G.C, rows = G.A * G.B;
    r.odd = (C & 1) != 0;
    r.M = r.odd ? C : C / 2;
    r.L = c2r_lines(r.M);
    r.ncomp = job.ncomp;
    r.RPC = max(1, r.L / r.ncomp);
    r.r0 = bw.tile * r.RPC;
    r.nl = min(r.RPC, rows - r.r0);
    r.comp0 = r.ncomp == 1 ? bw.comp : 0;
    return r;
}

// spectrum rows: raw X[k], k <= M, into slot k * LDI + cc * nl + l
__device__ __forceinline__ void c2r_prefetch(const SimDev& G, const BlockWork bw, const RowC2RJob& job, float2* buf, int t) {
    if (!gate_open(G, job.gate, bw.comp, t)) return;
    const RowTile r = c2r_tile(G, job, bw);
    const int LDI = r.L + 1;
    const int Mx = r.odd ? G.Ch : r.M + 1;   // staged bins per row
    for (int cc = 0; cc < r.ncomp; ++cc) {
        const float2* X = G.spec[job.spec_in + r.comp0 + cc] + (long long)r.r0 * G.Cp;
        for (int w = threadIdx.x; w < r.nl * Mx; w += blockDim.x) {
            const int l = w / Mx, k = w - l * Mx;
            cp_async8(buf + k * LDI + cc * r.nl + l, X + (long long)l * G.Cp + k);
        }
    }
}

__device__ __forceinline__ void c2r_stage_aux(const SimDev& S, const AuxPlan& a, const RowTile& r, float* aux) {
    const int C = S.C;
    const int rowsz = r.RPC * C;
    for (int f = 0; f < AX_COUNT; ++f)
        if (a.src[f]) stage_rows(aux + a.slot[f] * rowsz, a.src[f] + (long long)r.r0 * C, r.nl, C);
}

// epilogue at one grid point; staged inputs come from `av(field)` (the value of that field here)
template <class AV>
__device__ __forceinline__ void epi_point(const SimDev& S, const RowC2RJob& job, int comp0, int ncomp, long long i,
                                          int ca, int cb, int cc, const float* d, AV av, const AdjTapeEntry* te,
                                          float sgain) {
    auto coord = [&](int ax) { const int L = ax + 3 - S.dim; return L == 0 ? ca : (L == 1 ? cb : cc); };
    auto c2_at = [&]() { return S.c2.ptr ? av(AX_C2) : S.c2.s; };
    auto rho0_at = [&]() { return S.rho0.ptr ? av(AX_RHO0) : S.rho0.s; };
    auto eos = [&](float rs, float divterm) {   // p = c0^2 (rho + tau rho0 divU + B/A rho^2/(2 rho0))
        float e = rs;
        if (S.absorb == 1) e = e + (S.tau.ptr ? av(AX_TAU) : S.tau.s) * divterm;
        if (S.nonlinear) e = e + (S.bona.ptr ? av(AX_BONA) : S.bona.s) * (rs * rs) / (2.f * rho0_at());
        return c2_at() * e;
    };
    switch (job.epi) {
        case EPI_STORE:
            for (int o = 0; o < ncomp; ++o) field_ptr(S, job.out_field, comp0 + o)[i] = d[o];
            break;
        case EPI_VEL: {  // u = pml_sg (pml_sg u - dt/rho_sg dp)   (KSpaceFirstOrder.swift:453-454)
            const int a = comp0;
            const float sg = __ldg(S.ax[a].pml_sg + coord(a));
            const float dtor = S.dtor[a].ptr ? av(AX_F1) : S.dtor[a].s;
            S.u[a][i] = sg * (sg * av(AX_F0) - dtor * d[0]);
            break;
        }
        case EPI_VEL_INIT: {  // u = (dt/rho_sg / 2) dp0   (KSpaceFirstOrder.swift:519-520)
            const int a = comp0;
            const float dtor = S.dtor[a].ptr ? av(AX_F1) : S.dtor[a].s;
            S.u[a][i] = (dtor / 2.f) * d[0];
            break;
        }
        case EPI_ADD_U:
            S.u[comp0][i] = av(AX_F0) + d[0];
            break;
        case EPI_DEN:
        case EPI_DEN_SRC: {  // KSpaceFirstOrder.swift:457-465 (+ EoS when pointwise)
            const float r0v = rho0_at();
            float nl = 1.f;
            if (S.nonlinear) {
                float rp = 0.f;
                for (int a = 0; a < S.dim; ++a) rp = a == 0 ? av(AX_F0) : rp + av(AX_F0 + a);
                nl = (2.f * rp + r0v) / r0v;
            }
            const float dtr = S.dt * r0v;   // dt * rho0 in FP32, as KSpaceFirstOrder.swift:400
            float rs = 0.f, dv = 0.f;
            for (int a = 0; a < S.dim; ++a) {
                const float pm = __ldg(S.ax[a].pml + coord(a));
                const float mass = S.nonlinear ? dtr * d[a] * nl : dtr * d[a];
                float r = pm * (pm * av(AX_F0 + a) - mass);
                // precorrected additive pressure source (SimDev::psrc_q)
                if (sgain != 0.f) r = r + (sgain * __ldg(S.psrc_q + i)) * S.ax[a].inv_d;
                S.rho[a][i] = r;
                if (te && (S.nonlinear || S.adj_gr)) te->dd[a][i] = d[a];   // the adjoint's recompute keeps d_a
                rs = a == 0 ? r : rs + r;
                dv = a == 0 ? d[a] : dv + d[a];
            }
            S.rho_sum[i] = rs;
            float divterm = 0.f;
            if (S.absorb >= 1) {
                divterm = r0v * dv;
                S.div_term[i] = divterm;
                if (te && S.absorb == 1) te->div[i] = divterm;
            }
            if (S.eos_pointwise) {
                const float pv = eos(rs, divterm);
                S.p[i] = pv;
                if (te) { te->s[i] = rs; te->p[i] = pv; }
            }
            break;
        }
        case EPI_ADD_RHO: {  // additive p source, k-space corrected (KSpaceFirstOrder.swift:167-172)
            float rs = 0.f;
            for (int a = 0; a < S.dim; ++a) {
                const float r = av(AX_F0 + a) + d[0] * S.ax[a].inv_d;
                S.rho[a][i] = r;
                rs = a == 0 ? r : rs + r;
            }
            S.rho_sum[i] = rs;
            if (S.eos_pointwise) {
                const float pv = eos(rs, S.absorb == 1 ? av(AX_ETA) : 0.f);
                S.p[i] = pv;
                if (te) { te->s[i] = rs; te->p[i] = pv; }
            }
            break;
        }
        case EPI_EOS_ABS: {  // power-law absorption / dispersion (KSpaceFirstOrder.swift:836-845)
            const float rs = av(AX_F0);
            float term = (S.tau.ptr ? av(AX_TAU) : S.tau.s) * d[0];
            if (S.absorb == 3) term = term - (S.eta.ptr ? av(AX_ETA) : S.eta.s) * d[1];
            float e = rs + term;
            if (S.nonlinear) e = e + (S.bona.ptr ? av(AX_BONA) : S.bona.s) * (rs * rs) / (2.f * rho0_at());
            S.p[i] = c2_at() * e;
            if (te) {   // the adjoint's recompute keeps p, S and A2(S)
                te->p[i] = c2_at() * e;
                te->s[i] = rs;
                if (S.absorb == 3) te->q2[i] = d[1];
            }
            break;
        }
        default: break;
    }
}

template <int MT>
__device__ __forceinline__ void c2r_compute(const SimDev& S, const BlockWork bw, const RowC2RJob& job, const AdjTapeEntry* te, float2* buf,
                                            float2* tmp, const float* aux, const AuxPlan& a, int t) {
    constexpr bool FIX = MT > 0;
    constexpr int LT = FIX ? c2r_lines(MT) : 1;
    const RowTile r = c2r_tile(S, job, bw);
    const int C = S.C;
    const int M = FIX ? MT : r.M;
    const int L = FIX ? LT : r.L;
    const int LDI = L + 1;
    const int nl = r.nl, ncomp = r.ncomp, lines = nl * ncomp;

    // Hermitian pre-processing in place, a pair (k, M-k) per work item:
    // Z'[k] = (X[k] + conj X[M-k]) + i exp(+2 pi i k / C) (X[k] - conj X[M-k]), real part at k = 0, M
    if (!r.odd) {
        const int npair = M / 2 + 1;
        for (int w = threadIdx.x; w < lines * npair; w += blockDim.x) {
            const int line = w / npair, k = w - line * npair;
            const int km = M - k;
            float2 a0 = buf[k * LDI + line], b0 = buf[km * LDI + line];
            if (k == 0) { a0.y = 0.f; b0.y = 0.f; }
            const float2 s = make_float2(a0.x + b0.x, a0.y - b0.y);
            const float2 dd = make_float2(a0.x - b0.x, a0.y + b0.y);
            const float2 e = cmulc(dd, __ldg(S.row_tw + k));
            buf[k * LDI + line] = make_float2(s.x - e.y, s.y + e.x);
            if (k != 0 && km != k) {
                // the partner bin: X[M-k] with conj X[k]
                const float2 s2 = make_float2(b0.x + a0.x, b0.y - a0.y);
                const float2 d2 = make_float2(b0.x - a0.x, b0.y + a0.y);
                const float2 e2 = cmulc(d2, __ldg(S.row_tw + km));
                buf[km * LDI + line] = make_float2(s2.x - e2.y, s2.y + e2.x);
            }
        }
    } else {
        // odd C: rebuild the full spectrum from the half (slots >= Ch mirror conj X[C-k])
        for (int w = threadIdx.x; w < lines * M; w += blockDim.x) {
            const int line = w / M, k = w - line * M;
            if (k >= S.Ch) continue;
            float2 v = buf[k * LDI + line];
            if (k == 0) v.y = 0.f;
            tmp[k * LDI + line] = v;
            if (k > 0) tmp[(C - k) * LDI + line] = make_float2(v.x, -v.y);
        }
        __syncthreads();
        for (int w = threadIdx.x; w < lines * M; w += blockDim.x) {
            const int line = w / M, k = w - line * M;
            buf[k * LDI + line] = tmp[k * LDI + line];
        }
    }
    __syncthreads();
    const float2* Z;
    if constexpr (FIX) Z = fft_tile<MT, LT, LT + 1, true>(buf, tmp, S.plan_row.twn, lines);
    else Z = fft_lines<true>(buf, tmp, S.plan_row, lines, 1, LDI, true);

    cp_wait<1>();        // this tile's staged epilogue inputs have landed
    __syncthreads();
    const float sgain = job.epi == EPI_DEN_SRC ? psrc_gain(S, t) : 0.f;
    const int rowsz = r.RPC * C;
    const int B = S.B;
    for (int w = threadIdx.x; w < nl * M; w += blockDim.x) {
        const int l = w / M, m = w - l * M;
        const int row = r.r0 + l;
        const int ca = row / B, cb = row - ca * B;
        float d0[kMaxComp], d1[kMaxComp];
#pragma unroll
        for (int cc = 0; cc < kMaxComp; ++cc) {
            if (cc < ncomp) {
                const float2 z = Z[m * LDI + cc * nl + l];
                d0[cc] = z.x;
                d1[cc] = z.y;
            }
        }
        if (!r.odd) {
            const long long i0 = (long long)row * C + 2 * m;
            const int e0 = l * C + 2 * m;
            epi_point(S, job, r.comp0, ncomp, i0, ca, cb, 2 * m, d0,
                      [&](int f) { return aux[a.slot[f] * rowsz + e0]; }, te, sgain);
            epi_point(S, job, r.comp0, ncomp, i0 + 1, ca, cb, 2 * m + 1, d1,
                      [&](int f) { return aux[a.slot[f] * rowsz + e0 + 1]; }, te, sgain);
        } else {
            const int e0 = l * C + m;
            epi_point(S, job, r.comp0, ncomp, (long long)row * C + m, ca, cb, m, d0,
                      [&](int f) { return aux[a.slot[f] * rowsz + e0]; }, te, sgain);
        }
    }
}

template <int MT>
__global__ void __launch_bounds__(256) k_row_c2r(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                                 const BlockWork* __restrict__ map, int nmap, RowC2RJob job) {
    extern __shared__ __align__(16) float2 sm[];
    __shared__ SimDev S;
    int cur = -1;
    const int t = *d_t;
    const long long te = job.tile_elems;
    float2* tmp = sm + 2 * te;                                       // runtime-plan sizes only
    float* aux = reinterpret_cast<float*>(sm + (job.generic ? 3 : 2) * te);
    int idx = blockIdx.x;
    if (idx < nmap) { const BlockWork b = map[idx]; c2r_prefetch(sims[b.sim], b, job, sm, t); }
    cp_commit();
#pragma unroll 1
    for (int k = 0; idx < nmap; ++k, idx += gridDim.x) {
        const BlockWork bw = map[idx];
        use_sim(S, cur, sims, bw.sim);
        const bool open = gate_open(S, job.gate, bw.comp, t);
        const RowTile r = c2r_tile(S, job, bw);
        const AuxPlan a = aux_plan(S, job, r.comp0);
        if (open) c2r_stage_aux(S, a, r, aux);                       // epilogue inputs of tile k
        cp_commit();
        const int nidx = idx + gridDim.x;
        if (nidx < nmap) { const BlockWork b = map[nidx]; c2r_prefetch(sims[b.sim], b, job, sm + ((k + 1) & 1) * te, t); }
        cp_commit();
        cp_wait<2>();                                                // spectrum of tile k
        __syncthreads();
        if (open) c2r_compute<MT>(S, bw, job, job.tape ? S.tape + t : nullptr, sm + (k & 1) * te, tmp, aux, a, t);
        __syncthreads();
    }
    cp_wait<0>();
}

void init_c2r_attributes(int optin) {
#define KW_SET(m) set_max_smem((const void*)k_row_c2r<m>, optin);
    KW_FFT_SIZES(KW_SET)
#undef KW_SET
    set_max_smem((const void*)k_row_c2r<0>, optin);
}

void launch_row_c2r(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                    const RowC2RJob& job, size_t smem, int size_class) {
    if (nmap <= 0) return;
    switch (size_class) {
#define KW_CASE(m) \
    case m: k_row_c2r<m><<<persistent_grid((const void*)k_row_c2r<m>, smem, nmap), 256, smem, st>>>(d_sims, d_t, map, nmap, job); break;
        KW_FFT_SIZES(KW_CASE)
#undef KW_CASE
        default:
            k_row_c2r<0><<<persistent_grid((const void*)k_row_c2r<0>, smem, nmap), 256, smem, st>>>(d_sims, d_t, map, nmap, job);
            break;
    }
}

}  // namespace kw
