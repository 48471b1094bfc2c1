// kw_pass_colop.cu — the operator column pass: the last forward pass of a spectral job (along A in
// 3D, along B in 2D) for the register-plan lengths (has_colop: N = 16 ... 1024).
//
// A CTA owns TW = colop_lines(N) consecutive spectrum columns; thread t of line l loads rows
// t + T r straight from HBM (consecutive lanes read consecutive columns), transforms forward
// (kw_fft_reg.cuh), multiplies by the radial table and 1/N, and transforms back with the
// intermediate product kept in registers. Outputs whose per-axis factor is along another axis share
// one inverse and take the factor on the way out; an output whose factor varies along the line
// gets its own inverse. With several outputs the product is parked in shared memory (each thread
// its own slots) so that only one line's worth of registers is live. Many small CTAs per SM keep
// enough loads in flight. The fan-in variant sums H_c X_c over several inputs into one output
// with one inverse.
#include "kw_fft_reg.cuh"
#include "kw_pass_common.cuh"

namespace kw {

// Variants (N, R1, MINB) of the operator pass: R1 values per thread (so N / R1 threads per line and
// colop_tile(N, R1) lines per CTA) and a launch bound of MINB resident CTAs per SM (0: the
// compiler's register choice). The first variant of each length is the default: three CTAs per SM
// (85 registers) up to 256 points, the compiler's choice above. The autotuner (kw_tune.cpp) times
// the variants of a length on the job it is about to run and keeps the fastest.
#define KW_COLOP_VARIANTS(X)                                                                            \
    X(16, 4, 3) X(32, 8, 3) X(24, 12, 3) X(48, 12, 3)                                                   \
    X(64, 8, 3) X(64, 8, 4) X(64, 16, 3) X(64, 16, 2)                                                   \
    X(128, 16, 3) X(128, 16, 2) X(128, 8, 3) X(128, 8, 4)                                               \
    X(256, 16, 3) X(256, 16, 2) X(256, 8, 3) X(256, 8, 4)                                               \
    X(512, 16, 0) X(512, 16, 2) X(512, 8, 2) X(512, 8, 3) X(512, 8, 4)                                  \
    X(1024, 16, 0) X(1024, 16, 2) X(1024, 8, 2) X(1024, 8, 3)                                           \
    X(96, 12, 3) X(96, 12, 2) X(96, 12, 4) X(192, 12, 3) X(192, 12, 2) X(192, 12, 4)                    \
    X(384, 12, 0) X(384, 12, 2) X(384, 12, 3) X(768, 12, 0) X(768, 12, 2) X(768, 12, 3)

template <int N, int R1V, int MINB>
__global__ void __launch_bounds__(256, MINB) k_colop(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                               const BlockWork* __restrict__ map, int nmap, ColJob job) {
    using P = RegPlan<N, R1V>;
    using Lay = ColLayout<P, N>;
    constexpr int R1 = P::R1, T = P::T, TW = P::LINES;
    __shared__ float2 sh[Lay::SLOTS];
    extern __shared__ __align__(16) float2 parked[];   // [R1][256] when the job has several outputs
    if (blockIdx.x >= nmap) return;
    const BlockWork bw = map[blockIdx.x];
    const SimDev& S = sims[bw.sim];
    if (!gate_open(S, job.gate, bw.comp, *d_t)) return;

    // the pass's lines are the columns of one plane (the layout axis before it has length 1)
    const bool axisA = job.layout_axis == 0;
    const int inner = axisA ? S.B * S.Cp : S.Cp;
    const int l = threadIdx.x % TW;
    const int t = threadIdx.x / TW;
    const int c = bw.tile * TW + l;
    const bool col_ok = c < inner;
    const long long base = col_ok ? c : 0;
    const float2* __restrict__ twn = axisA ? S.plan_a.twn : S.plan_b.twn;
    const int comp_in = job.fanout ? 0 : bw.comp;
    const float2* in = S.spec[job.spec_in + comp_in] + base;
    // the radial table of this thread's bins is copied into its own shared-memory slots while the
    // spectrum loads and the forward transform run (behind the parked product, if any)
    const int rad = (comp_in == 0 ? job.op[0] : (comp_in == 1 ? job.op[1] : job.op[2])).radial;
    float* tsl = reinterpret_cast<float*>(parked + (job.fanout && job.nout > 1 ? R1 * 256 : 0)) + threadIdx.x;
    if (rad != RT_NONE && col_ok) {
        const float* tab = S.radial[rad] + base;
#pragma unroll
        for (int r = 0; r < R1; ++r) cp_async4(tsl + r * 256, tab + (long long)(t + T * r) * inner);
    }
    cp_commit();

    float2 v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) v[r] = col_ok ? in[(long long)(t + T * r) * inner] : make_float2(0.f, 0.f);

    FftReg<N, P, false, Lay>::run(v, sh, t, l, twn);          // v[m] = X(row t + T m)
    int kb = 0, kc = c;
    if (axisA) { kb = c / S.Cp; kc = c - kb * S.Cp; }
    const bool bin_ok = col_ok && kc < S.Ch;
    const int pass_ref_axis = (axisA ? 0 : 1) - (3 - S.dim);
    const int nouts = job.fanout ? job.nout : 1;
    auto op_of = [&](int oc) { return oc == 0 ? job.op[0] : (oc == 1 ? job.op[1] : job.op[2]); };
    auto out_comp = [&](int oo) { return job.fanout ? oo : bw.comp; };
    auto factor_vec = [&](const OpSpec& op) -> const float2* {
        if (op.axis_op == AO_NONE) return nullptr;
        const AxisDev& ax = S.ax[op.axis];
        return op.axis_op == AO_DPOS ? ax.dpos : (op.axis_op == AO_DNEG ? ax.dneg : ax.colloc);
    };
    auto along = [&](const OpSpec& op) { return op.axis_op != AO_NONE && op.axis == pass_ref_axis; };
    // X * radial / N: the factor common to every output (padding bins are never stored: they stay zero)
    const float inv_n = S.inv_n;
    cp_wait<0>();
#pragma unroll
    for (int m = 0; m < R1; ++m) {
        float f = inv_n;
        if (rad != RT_NONE && bin_ok) f *= tsl[m * 256];
        v[m] = bin_ok ? cscale(v[m], f) : make_float2(0.f, 0.f);
    }
    // H_o = F_o(k_a) kappa / N. A factor F_o along another axis is constant along the line, so
    // it commutes with the inverse: those outputs share one inverse and take F_o on the way out.
    // With several outputs the product is parked in shared memory (this thread's own slots) so
    // that only one line's worth of registers is live.
    bool shared = false;
    for (int oo = 0; oo < nouts; ++oo) shared |= !along(op_of(out_comp(oo)));
    const bool park = nouts > 1;
    if (park) {
#pragma unroll
        for (int m = 0; m < R1; ++m) parked[m * 256 + threadIdx.x] = v[m];
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
    for (int oo = 0; oo < nouts; ++oo) {   // outputs whose factor varies along the line
        const int oc = out_comp(oo);
        const OpSpec op = op_of(oc);
        if (!along(op)) continue;
        const float2* fv = factor_vec(op);
        if (park) {
#pragma unroll
            for (int m = 0; m < R1; ++m) v[m] = parked[m * 256 + threadIdx.x];
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


// fan-in operator pass: sum_c H_c X_c over job.fanin inputs with one inverse transform (the
// adjoint's lambda_p = sum_a D-_a w_a); the running sum is kept in this thread's shared-memory slots
template <int N>
__global__ void __launch_bounds__(256, 2) k_colop_fanin(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                                        const BlockWork* __restrict__ map, int nmap, ColJob job) {
    using P = RegPlan<N, reg_r1(N)>;
    using Lay = ColLayout<P, N>;
    constexpr int R1 = P::R1, T = P::T, TW = P::LINES;
    __shared__ float2 sh[Lay::SLOTS];
    extern __shared__ __align__(16) float2 parked[];   // [R1][256]
    if (blockIdx.x >= nmap) return;
    const BlockWork bw = map[blockIdx.x];
    const SimDev& S = sims[bw.sim];
    if (!gate_open(S, job.gate, bw.comp, *d_t)) return;
    const bool axisA = job.layout_axis == 0;
    const int inner = axisA ? S.B * S.Cp : S.Cp;
    const int l = threadIdx.x % TW;
    const int t = threadIdx.x / TW;
    const int c = bw.tile * TW + l;
    const bool col_ok = c < inner;
    const long long base = col_ok ? c : 0;
    const float2* __restrict__ twn = axisA ? S.plan_a.twn : S.plan_b.twn;
    auto op_of = [&](int oc) { return oc == 0 ? job.op[0] : (oc == 1 ? job.op[1] : job.op[2]); };
    auto factor_vec = [&](const OpSpec& op) -> const float2* {
        if (op.axis_op == AO_NONE) return nullptr;
        const AxisDev& ax = S.ax[op.axis];
        return op.axis_op == AO_DPOS ? ax.dpos : (op.axis_op == AO_DNEG ? ax.dneg : ax.colloc);
    };
    const int pass_ref_axis = (axisA ? 0 : 1) - (3 - S.dim);
    // fan-in: sum_c H_c X_c with one inverse transform (the adjoint's lambda_p = sum_a D-_a w_a);
    // the running sum is kept in this thread's shared-memory slots
    int kb = 0, kc = c;
    if (axisA) { kb = c / S.Cp; kc = c - kb * S.Cp; }
    const bool bin_ok = col_ok && kc < S.Ch;
    float2 v[R1];
#pragma unroll 1
    for (int ci = 0; ci < job.fanin; ++ci) {
        const float2* inc = S.spec[job.spec_in + ci] + base;
#pragma unroll
        for (int r = 0; r < R1; ++r) v[r] = col_ok ? inc[(long long)(t + T * r) * inner] : make_float2(0.f, 0.f);
        FftReg<N, P, false, Lay>::run(v, sh, t, l, twn);
        const OpSpec op = op_of(ci);
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
            parked[m * 256 + threadIdx.x] = ci == 0 ? y : cadd(parked[m * 256 + threadIdx.x], y);
        }
    }
#pragma unroll
    for (int m = 0; m < R1; ++m) v[m] = parked[m * 256 + threadIdx.x];
    FftReg<N, P, true, Lay>::run(v, sh, t, l, twn);
    float2* out = S.spec[job.spec_out] + base;
    if (bin_ok) {
#pragma unroll
        for (int m = 0; m < R1; ++m) out[(long long)(t + T * m) * inner] = v[m];
    }
    return;
}

// dynamic shared memory: the parked product (several outputs, or the fan-in sum) and the radial
// table slots
static size_t colop_park_bytes(const ColJob& job, int r1) {
    const bool park = job.fanin || (job.fanout && job.nout > 1);
    const bool table = !job.fanin && (job.op[0].radial != RT_NONE || job.op[1].radial != RT_NONE || job.op[2].radial != RT_NONE);
    return (size_t)r1 * 256 * ((park ? sizeof(float2) : 0) + (table ? sizeof(float) : 0));
}

void init_colop_attributes(int optin) {
#define KW_SET(NN, RR, MB) set_max_smem((const void*)k_colop<NN, RR, MB>, optin);
    KW_COLOP_VARIANTS(KW_SET)
#undef KW_SET
#define KW_SET(n) set_max_smem((const void*)k_colop_fanin<n>, optin);
    KW_COLOP_SIZES(KW_SET)
#undef KW_SET
}

int colop_variants(int n, ColopVariant* out, int max) {
    int k = 0;
#define KW_ADD(NN, RR, MB) \
    if (n == NN && k < max) out[k++] = ColopVariant{RR, MB};
    KW_COLOP_VARIANTS(KW_ADD)
#undef KW_ADD
    return k;
}

void launch_colop(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                  const ColJob& job, int n, ColopVariant v) {
    if (nmap <= 0) return;
    if (job.fanin) {   // one variant (the adjoint's fan-in sum)
        switch (n) {
#define KW_CASE(n) \
    case n: k_colop_fanin<n><<<nmap, 256, colop_park_bytes(job, reg_r1(n)), st>>>(d_sims, d_t, map, nmap, job); break;
            KW_COLOP_SIZES(KW_CASE)
#undef KW_CASE
            default: break;
        }
        return;
    }
#define KW_CASE(NN, RR, MB)                                                                                 \
    if (n == NN && v.r1 == RR && v.minb == MB) {                                                            \
        k_colop<NN, RR, MB><<<nmap, 256, colop_park_bytes(job, RR), st>>>(d_sims, d_t, map, nmap, job);     \
        return;                                                                                             \
    }
    KW_COLOP_VARIANTS(KW_CASE)
#undef KW_CASE
}

}  // namespace kw
