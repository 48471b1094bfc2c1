// kw_pass_col.cu — column pass: C2C along a strided layout axis (B, then A) on tiles of
// contiguous spectrum columns. MODE = COL_FWD / COL_INV transforms in place; MODE = COL_FWD_OP_INV
// (the last forward pass) transforms forward, multiplies by the k-space operator(s) and 1/N, and
// transforms back along the same axis while the tile is on chip, writing one or several outputs.
#include "kw_pass_common.cuh"

namespace kw {

template <int MODE>
__host__ __device__ constexpr int col_tw(int n) { return MODE == COL_FWD_OP_INV ? col_lines_op(n) : col_lines(n); }

// resident CTAs per SM asked of the register allocator for the operator pass (two transforms)
#ifndef KW_MINB_OP
#define KW_MINB_OP 2
#endif

struct ColGeom {
    int n, inner, TW, o, c0, ncols;
    long long obase;
};

template <int MODE>
__device__ __forceinline__ ColGeom col_geom(const SimDev& G, const ColJob& job, int tile) {
    ColGeom g;
    const bool axisA = job.layout_axis == 0;
    g.n = axisA ? G.A : G.B;
    g.inner = axisA ? G.B * G.Cp : G.Cp;
    g.TW = col_tw<MODE>(g.n);
    const int nchunks = (g.inner + g.TW - 1) / g.TW;
    g.o = tile / nchunks;
    g.c0 = (tile - g.o * nchunks) * g.TW;
    g.ncols = min(g.TW, g.inner - g.c0);
    g.obase = (long long)g.o * g.n * g.inner + g.c0;
    return g;
}

// stage the tile (and, for an operator pass, the radial table under it)
template <int MODE>
__device__ __forceinline__ void col_prefetch(const SimDev& G, const BlockWork bw, const ColJob& job, float2* buf,
                                             float* rbuf, int t) {
    if (!gate_open(G, job.gate, bw.comp, t)) return;
    const ColGeom g = col_geom<MODE>(G, job, bw.tile);
    const int comp_in = job.fanout ? 0 : bw.comp;
    const float2* in = G.spec[job.spec_in + comp_in] + g.obase;
    const int TW = g.TW, half = TW / 2;
    // pairs of columns: 16-byte copies (inner, c0 and TW are even, spectra 256-byte aligned)
    for (int w = threadIdx.x; w < g.n * half; w += blockDim.x) {
        const int i = w / half, l2 = (w - i * half) * 2;
        float2* d = buf + i * TW + l2;
        if (l2 < g.ncols) cp_async16(d, in + (long long)i * g.inner + l2);
        else { d[0] = make_float2(0.f, 0.f); d[1] = make_float2(0.f, 0.f); }
    }
    // the radial table of this tile's operator (all outputs of a fan-out share one); pairs of
    // columns as 8-byte copies (inner, c0 and TW are even)
    const int rad = job.op[job.fanout ? 0 : bw.comp].radial;
    if (MODE == COL_FWD_OP_INV && rad != RT_NONE) {
        const float* tab = G.radial[rad] + g.obase;
        for (int w = threadIdx.x; w < g.n * half; w += blockDim.x) {
            const int i = w / half, l2 = (w - i * half) * 2;
            if (l2 < g.ncols) cp_async8(rbuf + i * TW + l2, tab + (long long)i * g.inner + l2);
        }
    }
}

template <int NT, int MODE, bool INV>
__device__ __forceinline__ float2* col_fft(float2* a, float2* b, const FFTPlanDev& pl, int TW) {
    if constexpr (NT > 0) {
        constexpr int LT = col_tw<MODE>(NT);
        return fft_tile<NT, LT, LT, INV>(a, b, pl.twn, TW);
    } else {
        return fft_lines<INV>(a, b, pl, TW, 1, TW, true);
    }
}

template <int NT, int MODE>
__device__ __forceinline__ void col_store(const SimDev& S, const ColGeom& g, float2* out, const float2* R) {
    const int n = NT > 0 ? NT : g.n;
    const int TW = g.TW, half = TW / 2;
    for (int w = threadIdx.x; w < n * half; w += blockDim.x) {
        const int i = w / half, l2 = (w - i * half) * 2;
        if (l2 < g.ncols)
            *reinterpret_cast<float4*>(out + (long long)i * g.inner + l2) = *reinterpret_cast<const float4*>(R + i * TW + l2);
    }
}

template <int NT, int MODE>
__device__ __forceinline__ void col_compute(const SimDev& S, const BlockWork bw, const ColJob& job, float2* X,
                                            const float* R, float2* P, float2* Q) {
    const bool axisA = job.layout_axis == 0;
    const ColGeom g = col_geom<MODE>(S, job, bw.tile);
    const int n = NT > 0 ? NT : g.n;
    const int TW = g.TW;
    const FFTPlanDev& pl = axisA ? S.plan_a : S.plan_b;
    const int comp_in = job.fanout ? 0 : bw.comp;

    if constexpr (MODE != COL_FWD_OP_INV) {
        const float2* Rr = col_fft<NT, MODE, MODE == COL_INV>(X, P, pl, TW);
        col_store<NT, MODE>(S, g, S.spec[job.spec_in + comp_in] + g.obase, Rr);
    } else {
        // H_o = F_o(k_a) kappa(|k|) / N. A per-axis factor F_o whose axis is not this pass's axis is
        // constant along every line of the tile, so it commutes with the inverse transform along
        // the line: all such outputs share one inverse of kappa X / N and take their factor on the
        // way out. Only an output whose factor varies along the line needs its own inverse.
        float2* F = col_fft<NT, MODE, false>(X, P, pl, TW);
        float2* W = F == X ? P : X;   // work buffer for the operator product
        const int nouts = job.fanout ? job.nout : 1;
        const int pass_ref_axis = (axisA ? 0 : 1) - (3 - S.dim);   // reference axis of this pass
        const int rad = job.op[job.fanout ? 0 : bw.comp].radial;
        auto factor_vec = [&](const OpSpec& op) -> const float2* {
            if (op.axis_op == AO_NONE) return nullptr;
            const AxisDev& ax = S.ax[op.axis];
            return op.axis_op == AO_DPOS ? ax.dpos : (op.axis_op == AO_DNEG ? ax.dneg : ax.colloc);
        };
        auto column_k = [&](const OpSpec& op, int c) {   // wavenumber index of a column along op.axis
            int kb, kc;
            if (axisA) { kb = c / S.Cp; kc = c - kb * S.Cp; }
            else { kb = 0; kc = c; }
            return axis_index(S, op.axis, 0, kb, kc);
        };
        // fill W = f(i, col) F / N and inverse-transform it (returns the buffer holding the result)
        auto run = [&](const float2* alongv) {
            for (int w = threadIdx.x; w < n * TW; w += blockDim.x) {
                const int i = w / TW, l = w - i * TW;
                const int c = g.c0 + l;
                float2 v = make_float2(0.f, 0.f);
                int kc = axisA ? c - (c / S.Cp) * S.Cp : c;
                if (l < g.ncols && kc < S.Ch) {
                    float2 f = make_float2(S.inv_n, 0.f);
                    if (alongv) f = cscale(__ldg(alongv + i), S.inv_n);
                    if (rad != RT_NONE) f = cscale(f, R[w]);
                    v = cmul(F[w], f);
                }
                W[w] = v;
            }
            __syncthreads();
            return col_fft<NT, MODE, true>(W, Q, pl, TW);
        };
        // store T, multiplied by a per-column factor (a factor along another axis) when given
        auto column_kc = [&](int c) { return axisA ? c - (c / S.Cp) * S.Cp : c; };
        auto store_scaled = [&](int oc, const float2* T, const float2* colv, const OpSpec& op) {
            float2* out = S.spec[job.spec_out + oc] + g.obase;
            const int half = TW / 2;
            for (int w = threadIdx.x; w < n * half; w += blockDim.x) {
                const int i = w / half, l2 = (w - i * half) * 2;
                if (l2 >= g.ncols) continue;
                float2 a0 = T[i * TW + l2], a1 = T[i * TW + l2 + 1];
                if (colv) {   // padding columns (kc >= Ch) hold zeros and keep them
                    const int c = g.c0 + l2;
                    if (column_kc(c) < S.Ch) a0 = cmul(a0, __ldg(colv + column_k(op, c)));
                    if (column_kc(c + 1) < S.Ch) a1 = cmul(a1, __ldg(colv + column_k(op, c + 1)));
                }
                *reinterpret_cast<float4*>(out + (long long)i * g.inner + l2) = make_float4(a0.x, a0.y, a1.x, a1.y);
            }
        };
        const float2* T0 = nullptr;
        for (int oo = 0; oo < nouts; ++oo) {          // outputs whose factor is constant along the line
            const int oc = job.fanout ? oo : bw.comp;
            const OpSpec op = job.op[oc];
            if (op.axis_op != AO_NONE && op.axis == pass_ref_axis) continue;
            if (!T0) T0 = run(nullptr);
            store_scaled(oc, T0, factor_vec(op), op);
        }
        if (T0) __syncthreads();
        for (int oo = 0; oo < nouts; ++oo) {          // outputs whose factor varies along the line
            const int oc = job.fanout ? oo : bw.comp;
            const OpSpec op = job.op[oc];
            if (!(op.axis_op != AO_NONE && op.axis == pass_ref_axis)) continue;
            const float2* T = run(factor_vec(op));
            store_scaled(oc, T, nullptr, op);
            __syncthreads();
        }
    }
}

// shared memory: [tile0][tile1] (+ [radial0|radial1][W] for the operator pass)
//                (+ one ping-pong tile for the runtime plan)
template <int NT, int MODE>
__global__ void __launch_bounds__(256, (MODE == COL_FWD_OP_INV ? KW_MINB_OP : 1)) k_col(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                             const BlockWork* __restrict__ map, int nmap, ColJob job) {
    extern __shared__ __align__(16) float2 sm[];
    __shared__ SimDev S;
    int cur = -1;
    const int t = *d_t;
    const long long te = job.tile_elems;
    constexpr bool OP = MODE == COL_FWD_OP_INV;
    float* rad = reinterpret_cast<float*>(sm + 2 * te);
    float2* P = sm + (OP ? 3 : 2) * te;
    float2* Q = P + te;
    int idx = blockIdx.x;
    if (idx < nmap) { const BlockWork b = map[idx]; col_prefetch<MODE>(sims[b.sim], b, job, sm, rad, t); }
    cp_commit();
#pragma unroll 1
    for (int k = 0; idx < nmap; ++k, idx += gridDim.x) {
        const int nidx = idx + gridDim.x;
        if (nidx < nmap) {
            const BlockWork b = map[nidx];
            col_prefetch<MODE>(sims[b.sim], b, job, sm + ((k + 1) & 1) * te, rad + ((k + 1) & 1) * te, t);
        }
        cp_commit();
        cp_wait<1>();
        const BlockWork bw = map[idx];
        use_sim(S, cur, sims, bw.sim);
        if (gate_open(S, job.gate, bw.comp, t))
            col_compute<NT, MODE>(S, bw, job, sm + (k & 1) * te, rad + (k & 1) * te, P, Q);
        __syncthreads();
    }
    cp_wait<0>();
}

template <int MODE>
static void set_col_attrs(int optin) {
#define KW_SET(m) set_max_smem((const void*)k_col<m, MODE>, optin);
    KW_FFT_SIZES(KW_SET)
#undef KW_SET
    set_max_smem((const void*)k_col<0, MODE>, optin);
}

void init_col_attributes(int optin) {
    set_col_attrs<COL_FWD>(optin);
    set_col_attrs<COL_INV>(optin);
    set_col_attrs<COL_FWD_OP_INV>(optin);
    init_colop_attributes(optin);
    init_cola_attributes(optin);
    init_plane_attributes(optin);
}

template <int MODE>
static void launch_col_mode(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                            const ColJob& job, size_t smem, int size_class) {
    switch (size_class) {
#define KW_CASE(m)                                                                                                 \
    case m:                                                                                                        \
        k_col<m, MODE><<<persistent_grid((const void*)k_col<m, MODE>, smem, nmap), 256, smem, st>>>(d_sims, d_t, map, \
                                                                                                  nmap, job);      \
        break;
        KW_FFT_SIZES(KW_CASE)
#undef KW_CASE
        default:
            k_col<0, MODE><<<persistent_grid((const void*)k_col<0, MODE>, smem, nmap), 256, smem, st>>>(d_sims, d_t, map,
                                                                                                     nmap, job);
            break;
    }
}

void launch_col(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                const ColJob& job, size_t smem, int size_class) {
    if (nmap <= 0) return;
    if (job.mode == COL_FWD) launch_col_mode<COL_FWD>(st, d_sims, d_t, map, nmap, job, smem, size_class);
    else if (job.mode == COL_INV) launch_col_mode<COL_INV>(st, d_sims, d_t, map, nmap, job, smem, size_class);
    else launch_col_mode<COL_FWD_OP_INV>(st, d_sims, d_t, map, nmap, job, smem, size_class);
}

}  // namespace kw
