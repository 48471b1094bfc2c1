// kw_pass_cola.cu — persistent, double-buffered register column passes.
//
// A CTA of 256 threads owns TW = 256 / T consecutive spectrum columns per tile (T = N / R1 threads
// per line, thread t of line l holds rows t + T r, consecutive lanes on consecutive columns) and
// walks its share of the launch's tiles (tile k = blockIdx.x + j gridDim.x). While tile k is
// transformed, each thread has already issued the cp.async copies of its own R1 values of tile
// k + 1 into its own slots of the second landing buffer, so the HBM reads of the next tile overlap
// the transform, the operator product and the stores of this one. Because every thread only ever
// reads the slots it filled itself, the landing buffers need no barrier: cp.async.wait_group is
// enough. The shared-memory exchange of the transform (kw_fft_reg.cuh) is separate.
//
// Modes: in-place forward / inverse (the pass before and after the operator pass), the operator
// pass (forward, x radial table x per-axis factor / N, inverse; with fan-out several outputs from
// one input, the product parked in this tile's landing slots, which are free once read), and the
// fan-in operator pass (sum over the inputs of H_c X_c, one inverse). The radial table of the next
// tile is prefetched into L2 with the spectrum copies.
#include "kw_fft_reg.cuh"
#include "kw_pass_common.cuh"

namespace kw {

template <int N, int MODE>
__global__ void __launch_bounds__(256, 2) k_cola(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                                 const BlockWork* __restrict__ map, int nmap, ColJob job) {
    pdl_enter();
    using P = RegPlan<N, reg_r1(N)>;
    using Lay = ColLayout<P, N>;
    constexpr int R1 = P::R1, T = P::T, TW = P::LINES;
    constexpr bool OPM = MODE == CA_OP || MODE == CA_FANIN;
    __shared__ float2 sh[Lay::SLOTS];
    extern __shared__ __align__(16) float2 land[];   // [2][R1][256]: each thread's own slots
    const int tstep = *d_t;
    const int l = threadIdx.x % TW;
    const int t = threadIdx.x / TW;
    const bool axisA = job.layout_axis == 0;
    const int nsub = MODE == CA_FANIN ? job.fanin : 1;

    auto next_open = [&](int idx) {
        while (idx < nmap) {
            const BlockWork bw = map[idx];
            if (gate_open(sims[bw.sim], job.gate, bw.comp, tstep)) break;
            idx += gridDim.x;
        }
        return idx;
    };
    auto op_of = [&](int oc) { return oc == 0 ? job.op[0] : (oc == 1 ? job.op[1] : job.op[2]); };
    // tile geometry: lines of one plane (3D along B: plane o = the A index; otherwise one plane)
    auto column = [&](const SimDev& S, int tile, int& inner, long long& base, int& c) {
        inner = axisA ? S.B * S.Cp : S.Cp;
        const int nch = (inner + TW - 1) / TW;
        const int o = tile / nch;
        c = (tile - o * nch) * TW + l;
        base = (long long)o * N * inner + (c < inner ? c : 0);
    };
    auto in_comp = [&](const BlockWork& bw, int sub) { return MODE == CA_FANIN ? sub : (job.fanout ? 0 : bw.comp); };
    // copy this thread's values of unit (idx, sub) into landing buffer b (an empty group past the end)
    auto issue = [&](int idx, int sub, int b) {
        if (idx < nmap) {
            const BlockWork bw = map[idx];
            const SimDev& S = sims[bw.sim];
            int inner, c;
            long long base;
            column(S, bw.tile, inner, base, c);
            const float2* src = S.spec[job.spec_in + in_comp(bw, sub)] + base;
            float2* dst = land + b * (R1 * 256) + threadIdx.x;
            if (c < inner) {
#pragma unroll
                for (int r = 0; r < R1; ++r) cp_async8(dst + r * 256, src + (long long)(t + T * r) * inner);
                if constexpr (OPM) {
                    const int rad = op_of(MODE == CA_FANIN ? sub : (job.fanout ? 0 : bw.comp)).radial;
                    if (rad != RT_NONE) {
                        const float* tab = S.radial[rad] + base;
#pragma unroll
                        for (int r = 0; r < R1; ++r)
                            asm volatile("prefetch.global.L2 [%0];" ::"l"(tab + (long long)(t + T * r) * inner));
                    }
                }
            } else {
#pragma unroll
                for (int r = 0; r < R1; ++r) dst[r * 256] = make_float2(0.f, 0.f);
            }
        }
        cp_commit();
    };

    float2 acc[MODE == CA_FANIN ? R1 : 1];
    int idx = next_open(blockIdx.x), sub = 0, b = 0;
    issue(idx, 0, 0);
    while (idx < nmap) {
        int nidx = idx, nsb = sub + 1;
        if (nsb == nsub) {
            nidx = next_open(idx + gridDim.x);
            nsb = 0;
        }
        issue(nidx, nsb, b ^ 1);
        cp_wait<1>();   // this unit's copies (issued one unit earlier) have landed

        const BlockWork bw = map[idx];
        const SimDev& S = sims[bw.sim];
        int inner, c;
        long long base;
        column(S, bw.tile, inner, base, c);
        const bool col_ok = c < inner;
        int kb = 0, kc = c;
        if (axisA) { kb = c / S.Cp; kc = c - kb * S.Cp; }
        // padding bins (kc >= Ch) are never written: they stay zero
        const bool bin_ok = col_ok && kc < S.Ch;
        const float2* __restrict__ twn = axisA ? S.plan_a.twn : S.plan_b.twn;
        float2* lb = land + b * (R1 * 256) + threadIdx.x;

        float2 v[R1];
#pragma unroll
        for (int r = 0; r < R1; ++r) v[r] = lb[r * 256];

        if constexpr (MODE == CA_FWD || MODE == CA_INV) {
            FftReg<N, P, MODE == CA_INV, Lay>::run(v, sh, t, l, twn);
            float2* out = S.spec[job.spec_in + in_comp(bw, 0)] + base;
            if (bin_ok) {
#pragma unroll
                for (int m = 0; m < R1; ++m) out[(long long)(t + T * m) * inner] = v[m];
            }
        } else {
            FftReg<N, P, false, Lay>::run(v, sh, t, l, twn);   // v[m] = X(row t + T m)
            const int pass_ref_axis = (axisA ? 0 : 1) - (3 - S.dim);
            auto factor_vec = [&](const OpSpec& op) -> const float2* {
                if (op.axis_op == AO_NONE) return nullptr;
                const AxisDev& ax = S.ax[op.axis];
                return op.axis_op == AO_DPOS ? ax.dpos : (op.axis_op == AO_DNEG ? ax.dneg : ax.colloc);
            };
            if constexpr (MODE == CA_FANIN) {
                const OpSpec op = op_of(sub);
                const float2* fv = factor_vec(op);
                const bool alg = fv && op.axis == pass_ref_axis;
                float2 fc = make_float2(S.inv_n, 0.f);
                if (fv && !alg && bin_ok) fc = cscale(__ldg(fv + axis_index(S, op.axis, 0, kb, kc)), S.inv_n);
                const float* tab = op.radial != RT_NONE ? S.radial[op.radial] + base : nullptr;
#pragma unroll
                for (int m = 0; m < R1; ++m) {
                    float2 f = alg ? cscale(__ldg(fv + t + T * m), S.inv_n) : fc;
                    if (tab && bin_ok) f = cscale(f, __ldg(tab + (long long)(t + T * m) * inner));
                    const float2 y = bin_ok ? cmul(v[m], f) : make_float2(0.f, 0.f);
                    acc[m] = sub == 0 ? y : cadd(acc[m], y);
                }
                if (sub + 1 == nsub) {
#pragma unroll
                    for (int m = 0; m < R1; ++m) v[m] = acc[m];
                    FftReg<N, P, true, Lay>::run(v, sh, t, l, twn);
                    float2* out = S.spec[job.spec_out] + base;
                    if (bin_ok) {
#pragma unroll
                        for (int m = 0; m < R1; ++m) out[(long long)(t + T * m) * inner] = v[m];
                    }
                }
            } else {
                const int nouts = job.fanout ? job.nout : 1;
                auto out_comp = [&](int oo) { return job.fanout ? oo : bw.comp; };
                auto along = [&](const OpSpec& op) { return op.axis_op != AO_NONE && op.axis == pass_ref_axis; };
                const int rad = op_of(job.fanout ? 0 : bw.comp).radial;
                // X * radial / N: the factor common to every output
                const float* tab = rad != RT_NONE ? S.radial[rad] + base : nullptr;
#pragma unroll
                for (int m = 0; m < R1; ++m) {
                    float f = S.inv_n;
                    if (tab && bin_ok) f *= __ldg(tab + (long long)(t + T * m) * inner);
                    v[m] = bin_ok ? cscale(v[m], f) : make_float2(0.f, 0.f);
                }
                // H_o = F_o(k_a) kappa / N. A factor along another axis is constant along the line
                // and commutes with the inverse: those outputs share one inverse and take F_o on the
                // way out; an output whose factor varies along the line gets its own inverse, from
                // the product parked in this thread's landing slots.
                bool shared = false;
                for (int oo = 0; oo < nouts; ++oo) shared |= !along(op_of(out_comp(oo)));
                const bool park = nouts > 1;
                if (park) {
#pragma unroll
                    for (int m = 0; m < R1; ++m) lb[m * 256] = v[m];
                }
                if (shared) {
                    FftReg<N, P, true, Lay>::run(v, sh, t, l, twn);
                    for (int oo = 0; oo < nouts; ++oo) {
                        const int oc = out_comp(oo);
                        const OpSpec op = op_of(oc);
                        if (along(op)) continue;
                        const float2* fv = factor_vec(op);
                        float2 f = make_float2(1.f, 0.f);
                        if (fv && bin_ok) f = __ldg(fv + axis_index(S, op.axis, 0, kb, kc));
                        float2* out = S.spec[job.spec_out + oc] + base;
                        if (bin_ok) {
#pragma unroll
                            for (int m = 0; m < R1; ++m) out[(long long)(t + T * m) * inner] = cmul(v[m], f);
                        }
                    }
                }
                for (int oo = 0; oo < nouts; ++oo) {
                    const int oc = out_comp(oo);
                    const OpSpec op = op_of(oc);
                    if (!along(op)) continue;
                    const float2* fv = factor_vec(op);
                    if (park) {
#pragma unroll
                        for (int m = 0; m < R1; ++m) v[m] = lb[m * 256];
                    }
#pragma unroll
                    for (int m = 0; m < R1; ++m) v[m] = cmul(v[m], __ldg(fv + t + T * m));
                    FftReg<N, P, true, Lay>::run(v, sh, t, l, twn);
                    float2* out = S.spec[job.spec_out + oc] + base;
                    if (bin_ok) {
#pragma unroll
                        for (int m = 0; m < R1; ++m) out[(long long)(t + T * m) * inner] = v[m];
                    }
                }
            }
        }
        idx = nidx;
        sub = nsb;
        b ^= 1;
    }
    cp_wait<0>();
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
template <int N>
static constexpr size_t cola_land_bytes() { return (size_t)2 * reg_r1(N) * 256 * sizeof(float2); }

void init_cola_attributes(int optin) {
#define KW_SET(n)                                                     \
    set_max_smem((const void*)k_cola<n, CA_FWD>, optin);            \
    set_max_smem((const void*)k_cola<n, CA_INV>, optin);            \
    set_max_smem((const void*)k_cola<n, CA_OP>, optin);             \
    set_max_smem((const void*)k_cola<n, CA_FANIN>, optin);
    KW_COLOP_SIZES(KW_SET)
#undef KW_SET
}

template <int N, int MODE>
static void cola_launch(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                        const ColJob& job) {
    static int grid_cap = 0;
    if (!grid_cap) grid_cap = persistent_grid((const void*)k_cola<N, MODE>, cola_land_bytes<N>(), 1 << 30);
    const int grid = nmap < grid_cap ? nmap : grid_cap;
    launch_pdl(k_cola<N, MODE>, grid, 256, cola_land_bytes<N>(), st, d_sims, d_t, map, nmap, job);
}

void launch_cola(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                 const ColJob& job, int n) {
    if (nmap <= 0) return;
    const int mode = job.mode == COL_FWD ? CA_FWD : (job.mode == COL_INV ? CA_INV : (job.fanin ? CA_FANIN : CA_OP));
    switch (n) {
#define KW_CASE(n)                                                                 \
    case n:                                                                        \
        switch (mode) {                                                            \
            case CA_FWD: cola_launch<n, CA_FWD>(st, d_sims, d_t, map, nmap, job); break;     \
            case CA_INV: cola_launch<n, CA_INV>(st, d_sims, d_t, map, nmap, job); break;     \
            case CA_OP: cola_launch<n, CA_OP>(st, d_sims, d_t, map, nmap, job); break;       \
            default: cola_launch<n, CA_FANIN>(st, d_sims, d_t, map, nmap, job); break;       \
        }                                                                          \
        break;
        KW_COLOP_SIZES(KW_CASE)
#undef KW_CASE
        default: break;
    }
}

}  // namespace kw
