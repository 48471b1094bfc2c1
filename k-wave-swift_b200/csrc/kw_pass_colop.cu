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
#include "kw_async.cuh"
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

// The operator work of one tile after its spectrum is in registers (v[m] = X(row t + T m) of line
// l, not yet transformed): forward transform, x radial table (this thread's slots `tsl`, filled by
// cp.async) x 1/N, inverse transform(s), outputs stored. `sh` is the exchange buffer of the
// transforms, `parked` this thread's slots for the product when the job has several outputs.
template <int N, class P, class Lay, class Sync>
__device__ __forceinline__ void colop_body(const SimDev& S, const ColJob& job, int comp, float2 (&v)[P::R1], float2* sh,
                                           float2* parked, const float* tsl, int t, int l, int c, bool col_ok,
                                           long long base, int inner, bool axisA, int rad) {
    constexpr int R1 = P::R1, T = P::T;
    const float2* __restrict__ twn = axisA ? S.plan_a.twn : S.plan_b.twn;
    FftReg<N, P, false, Lay, Sync>::run(v, sh, t, l, twn);          // v[m] = X(row t + T m)
    int kb = 0, kc = c;
    if (axisA) { kb = c / S.Cp; kc = c - kb * S.Cp; }
    const bool bin_ok = col_ok && kc < S.Ch;
    const int pass_ref_axis = (axisA ? 0 : 1) - (3 - S.dim);
    const int nouts = job.fanout ? job.nout : 1;
    auto op_of = [&](int oc) { return oc == 0 ? job.op[0] : (oc == 1 ? job.op[1] : job.op[2]); };
    auto out_comp = [&](int oo) { return job.fanout ? oo : comp; };
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
    const int me = threadIdx.x;   // consumer thread index (the 256 threads of the tile)
    if (park) {
#pragma unroll
        for (int m = 0; m < R1; ++m) parked[m * 256 + me] = v[m];
    }
    if (shared) {
        FftReg<N, P, true, Lay, Sync>::run(v, sh, t, l, twn);
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
            for (int m = 0; m < R1; ++m) v[m] = parked[m * 256 + me];
        }
#pragma unroll
        for (int m = 0; m < R1; ++m) v[m] = cmul(v[m], __ldg(fv + t + T * m));
        FftReg<N, P, true, Lay, Sync>::run(v, sh, t, l, twn);
        float2* out = S.spec[job.spec_out + oc] + base;
        if (bin_ok) {
#pragma unroll
            for (int m = 0; m < R1; ++m) out[(long long)(t + T * m) * inner] = v[m];
        }
    }
}

// the radial table of this thread's bins into its own shared-memory slots (cp.async), overlapping
// the forward transform
template <int R1, int T>
__device__ __forceinline__ void colop_table(const SimDev& S, int rad, bool col_ok, long long base, int inner, int t,
                                            float* tsl) {
    if (rad != RT_NONE && col_ok) {
        const float* tab = S.radial[rad] + base;
#pragma unroll
        for (int r = 0; r < R1; ++r) cp_async4(tsl + r * 256, tab + (long long)(t + T * r) * inner);
    }
    cp_commit();
}

template <int N, int R1V, int MINB>
__global__ void __launch_bounds__(256, MINB) k_colop(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                               const BlockWork* __restrict__ map, int nmap, ColJob job) {
    pdl_enter();
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
    const int comp_in = job.fanout ? 0 : bw.comp;
    const float2* in = S.spec[job.spec_in + comp_in] + base;
    const int rad = (comp_in == 0 ? job.op[0] : (comp_in == 1 ? job.op[1] : job.op[2])).radial;
    float* tsl = reinterpret_cast<float*>(parked + (job.fanout && job.nout > 1 ? R1 * 256 : 0)) + threadIdx.x;
    colop_table<R1, T>(S, rad, col_ok, base, inner, t, tsl);
    float2 v[R1];
#pragma unroll
    for (int r = 0; r < R1; ++r) v[r] = col_ok ? in[(long long)(t + T * r) * inner] : make_float2(0.f, 0.f);
    colop_body<N, P, Lay, BlockSync>(S, job, bw.comp, v, sh, parked, tsl, t, l, c, col_ok, base, inner, axisA, rad);
}

// Persistent variant: each CTA walks the tile map with stride gridDim.x, and before transforming
// tile i it asks for tile i + 1's rows of the spectrum and of its radial table to be brought into
// L2 (cp.async.bulk.prefetch, one per row segment and thread; no registers or shared memory), so
// the loads of the next tile find them there. The tile's own work is k_colop's.
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}
template <int N, int R1V, int MINB>
__global__ void __launch_bounds__(256, MINB) k_colop_pf(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                                        const BlockWork* __restrict__ map, int nmap, ColJob job) {
    pdl_enter();
    using P = RegPlan<N, R1V>;
    using Lay = ColLayout<P, N>;
    constexpr int R1 = P::R1, T = P::T, TW = P::LINES;
    __shared__ float2 sh[Lay::SLOTS];
    extern __shared__ __align__(16) float2 parked[];   // [R1][256] when the job has several outputs
    const int tstep = *d_t;
    const bool axisA = job.layout_axis == 0;
    const int l = threadIdx.x % TW;
    const int t = threadIdx.x / TW;
    float* tsl = reinterpret_cast<float*>(parked + (job.fanout && job.nout > 1 ? R1 * 256 : 0)) + threadIdx.x;
    // the next tile of this CTA whose gate is open (nmap when none is left)
    auto next_open = [&](int idx) {
        for (; idx < nmap; idx += gridDim.x) {
            const BlockWork bw = map[idx];
            if (gate_open(sims[bw.sim], job.gate, bw.comp, tstep)) break;
        }
        return idx;
    };
    // tile idx's N row segments (TW columns, the last tile possibly fewer: a multiple of 4, so every
    // segment is a multiple of 16 bytes and starts 16-byte aligned)
    auto prefetch = [&](int idx) {
        const BlockWork bw = map[idx];
        const SimDev& S = sims[bw.sim];
        const int inner = axisA ? S.B * S.Cp : S.Cp;
        const int c0 = bw.tile * TW;
        const int w = min(TW, inner - c0);
        const int comp_in = job.fanout ? 0 : bw.comp;
        const float2* in = S.spec[job.spec_in + comp_in] + c0;
        const int rad = (comp_in == 0 ? job.op[0] : (comp_in == 1 ? job.op[1] : job.op[2])).radial;
        const float* tab = rad != RT_NONE ? S.radial[rad] + c0 : nullptr;
        for (int r = threadIdx.x; r < N; r += blockDim.x) {
            prefetch_l2(in + (long long)r * inner, (unsigned)w * 8u);
            if (tab) prefetch_l2(tab + (long long)r * inner, (unsigned)w * 4u);
        }
    };
    int idx = next_open(blockIdx.x);
    while (idx < nmap) {
        const int cur = idx;
        idx = next_open(idx + gridDim.x);
        if (idx < nmap) prefetch(idx);   // comes into L2 during the transforms below
        const BlockWork bw = map[cur];
        const SimDev& S = sims[bw.sim];
        const int inner = axisA ? S.B * S.Cp : S.Cp;
        const int c = bw.tile * TW + l;
        const bool col_ok = c < inner;
        const long long base = col_ok ? c : 0;
        const int comp_in = job.fanout ? 0 : bw.comp;
        const float2* in = S.spec[job.spec_in + comp_in] + base;
        const int rad = (comp_in == 0 ? job.op[0] : (comp_in == 1 ? job.op[1] : job.op[2])).radial;
        colop_table<R1, T>(S, rad, col_ok, base, inner, t, tsl);
        float2 v[R1];
#pragma unroll
        for (int r = 0; r < R1; ++r) v[r] = col_ok ? in[(long long)(t + T * r) * inner] : make_float2(0.f, 0.f);
        colop_body<N, P, Lay, BlockSync>(S, job, bw.comp, v, sh, parked, tsl, t, l, c, col_ok, base, inner, axisA, rad);
    }
}

// Dense column layout (no padding) for LINES >= 16: a half warp (16 lanes) touches one row of
// 16 consecutive values in every access of the transform, so rows need no padding to avoid bank
// conflicts; the TMA tile itself ([row][LINES] float2) is in this layout.
template <class P, int N>
struct ColLayoutDense {
    static constexpr int SLOTS = N * P::LINES;
    __device__ __forceinline__ static int at(int j, int l) { return j * P::LINES + l; }
};

// TMA-fed, warp-specialised operator pass along layout axis A (3D; the column lengths of the
// in-place TMA pass, R1 = 16): a persistent CTA of 8 consumer warps and one producer warp. The
// producer loads each tile (colr_lines(N) columns by the N rows) with one tensor copy into a ring
// of `ns` stages; the consumers take their values, run the forward transform, operator and
// inverse(s) with the stage itself as the exchange buffer, store the outputs and only then release
// the stage, so up to ns - 1 further tiles are in flight meanwhile. Bounded waits as in kw_pass_colp.cu.
template <int N>
__global__ void __launch_bounds__(288, 2) k_colop_tma(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                                      const BlockWork* __restrict__ map, int nmap, ColJob job, int ns,
                                                      int* __restrict__ err) {
    pdl_enter();
    using P = RegPlan<N, 16>;
    using Lay = ColLayoutDense<P, N>;
    constexpr int R1 = P::R1, T = P::T, TW = P::LINES;
    constexpr int STAGE = N * TW * 8;
    static_assert(TW >= 16, "dense layout needs 16 lines");
    extern __shared__ __align__(128) unsigned char smem[];
    const bool park_on = job.fanout && job.nout > 1;
    float2* parked = reinterpret_cast<float2*>(smem + ns * STAGE);
    float* tslots = reinterpret_cast<float*>(smem + ns * STAGE + (park_on ? R1 * 256 * 8 : 0));
    uint64_t* full = reinterpret_cast<uint64_t*>(reinterpret_cast<unsigned char*>(tslots) + R1 * 256 * 4);
    uint64_t* empty = full + ns;
    __shared__ volatile int abort;   // set by the consumers when one of their waits ran out
    if (threadIdx.x == 0) {
        abort = 0;
        for (int s2 = 0; s2 < ns; ++s2) {
            mbar_init(full + s2, 1);
            mbar_init(empty + s2, 8);
        }
        fence_barrier_init();
    }
    __syncthreads();
    const int tstep = *d_t;

    if (threadIdx.x >= 256) {
        // ---------------- producer ----------------
        if (threadIdx.x != 256) return;
        int k = 0;
        for (int idx = blockIdx.x; idx < nmap; idx += gridDim.x) {
            const BlockWork bw = map[idx];
            const SimDev& S = sims[bw.sim];
            if (!gate_open(S, job.gate, bw.comp, tstep)) continue;
            const int s = k % ns;
            if (k >= ns && !mbar_wait_or_abort(empty + s, ((k / ns) & 1) ^ 1, err, KE_TIMEOUT_EMPTY, &abort)) break;
            const int comp_in = job.fanout ? 0 : bw.comp;
            mbar_arrive_expect_tx(full + s, STAGE);
            tma_load_2d(smem + s * STAGE, S.tmaps + tmap_spec(job.spec_in + comp_in, 0), bw.tile * TW, 0, full + s);
            ++k;
        }
        // every issued copy must have landed before this CTA's shared memory is released
        for (int j = k > ns ? k - ns : 0; j < k; ++j) mbar_wait(full + j % ns, (j / ns) & 1, err, KE_TIMEOUT_DRAIN);
        return;
    }

    // ---------------- consumers ----------------
    const int l = threadIdx.x % TW;
    const int t = threadIdx.x / TW;
    const int lane = threadIdx.x & 31;
    float* tsl = tslots + threadIdx.x;
    int k = 0;
    for (int idx = blockIdx.x; idx < nmap; idx += gridDim.x) {
        const BlockWork bw = map[idx];
        const SimDev& S = sims[bw.sim];
        if (!gate_open(S, job.gate, bw.comp, tstep)) continue;
        const int s = k % ns;
        const int inner = S.B * S.Cp;
        const int c = bw.tile * TW + l;
        const bool col_ok = c < inner;
        const long long base = col_ok ? c : 0;
        const int comp_in = job.fanout ? 0 : bw.comp;
        const int rad = (comp_in == 0 ? job.op[0] : (comp_in == 1 ? job.op[1] : job.op[2])).radial;
        colop_table<R1, T>(S, rad, col_ok, base, inner, t, tsl);   // overlaps the wait and the transform
        const bool ok = mbar_wait(full + s, (k / ns) & 1, err, KE_TIMEOUT_FULL, S.wait_cycles);
        int all_ok;
        asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, 1, 256, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
                     : "=r"(all_ok) : "r"((unsigned)ok) : "memory");
        if (!all_ok) {
            cp_wait<0>();
            if (threadIdx.x == 0) abort = 1;
            return;
        }
        float2* stage = reinterpret_cast<float2*>(smem + s * STAGE);
        float2 v[R1];
#pragma unroll
        for (int r = 0; r < R1; ++r) v[r] = stage[(t + T * r) * TW + l];
        ConsumerSync::sync();   // every value is read before the transform reuses the stage
        colop_body<N, P, Lay, ConsumerSync>(S, job, bw.comp, v, stage, parked, tsl, t, l, c, col_ok, base, inner, true,
                                            rad);
        ConsumerSync::sync();   // the last exchange through the stage is done
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + s);
        ++k;
    }
}

// fan-in operator pass: sum_c H_c X_c over job.fanin inputs with one inverse transform (the
// adjoint's lambda_p = sum_a D-_a w_a); the running sum is kept in this thread's shared-memory slots
template <int N>
__global__ void __launch_bounds__(256, 2) k_colop_fanin(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                                        const BlockWork* __restrict__ map, int nmap, ColJob job) {
    pdl_enter();
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

// (N, R1, CTAs per SM) of the persistent L2-prefetching variant (minb = kColopPf - CTAs per SM)
#define KW_COLOP_PF(X) X(128, 16, 3) X(256, 16, 3) X(256, 16, 2) X(256, 8, 3) X(512, 16, 2) X(512, 8, 3) X(192, 12, 3) X(384, 12, 2)

void init_colop_attributes(int optin) {
#define KW_SET(NN, RR, MB) set_max_smem((const void*)k_colop<NN, RR, MB>, optin);
    KW_COLOP_VARIANTS(KW_SET)
#undef KW_SET
#define KW_SET(NN, RR, MB) set_max_smem((const void*)k_colop_pf<NN, RR, MB>, optin);
    KW_COLOP_PF(KW_SET)
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
#define KW_ADD(NN, RR, MB) \
    if (n == NN && k < max) out[k++] = ColopVariant{RR, kColopPf - MB};
    KW_COLOP_PF(KW_ADD)
#undef KW_ADD
    return k;
}

template <int N, int R1, int MB>
static void launch_colop_pf(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                            const ColJob& job) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    const size_t smem = colop_park_bytes(job, R1);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_colop_pf<N, R1, MB>, 256, smem) != cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    const int grid = nmap < per_sm * sms ? nmap : per_sm * sms;
    launch_pdl(k_colop_pf<N, R1, MB>, grid, 256, smem, st, d_sims, d_t, map, nmap, job);
}

// shared memory of the TMA-fed operator pass: `ns` stages, the parked product (several outputs),
// the radial table slots, the mbarriers; ns as large as two CTAs per SM allow (at most 4)
template <int N>
static void colop_tma_layout(const ColJob& job, int* ns, size_t* bytes) {
    constexpr size_t STAGE = (size_t)N * reg_lines(N, 16) * 8;
    const size_t fixed = (job.fanout && job.nout > 1 ? 16 * 256 * 8 : 0) + 16 * 256 * 4;
    const size_t budget = 113 * 1024 - 128;
    int k = (int)((budget - fixed) / (STAGE + 16));
    k = k < 2 ? 2 : (k > 4 ? 4 : k);
    *ns = k;
    *bytes = (size_t)k * STAGE + fixed + 16 * (size_t)k;
}

template <int N>
static void launch_colop_tma(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                             const ColJob& job, int* err) {
    int ns;
    size_t smem;
    colop_tma_layout<N>(job, &ns, &smem);
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    cudaFuncSetAttribute((const void*)k_colop_tma<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_colop_tma<N>, 288, smem) != cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    const int grid = nmap < per_sm * sms ? nmap : per_sm * sms;
    launch_pdl(k_colop_tma<N>, grid, 288, smem, st, d_sims, d_t, map, nmap, job, ns, err);
}

bool colop_tma_length(int n) { return n == 128 || n == 256; }

void launch_colop(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                  const ColJob& job, int n, ColopVariant v, int* err) {
    if (nmap <= 0) return;
    if (v.minb == kColopTma && !job.fanin) {
        if (n == 256) launch_colop_tma<256>(st, d_sims, d_t, map, nmap, job, err);
        else if (n == 128) launch_colop_tma<128>(st, d_sims, d_t, map, nmap, job, err);
        return;
    }
    if (v.minb <= kColopPf && !job.fanin) {
#define KW_CASE(NN, RR, MB)                                                  \
    if (n == NN && v.r1 == RR && v.minb == kColopPf - MB) {                  \
        launch_colop_pf<NN, RR, MB>(st, d_sims, d_t, map, nmap, job);        \
        return;                                                              \
    }
        KW_COLOP_PF(KW_CASE)
#undef KW_CASE
        return;
    }
    if (job.fanin) {   // one variant (the adjoint's fan-in sum)
        switch (n) {
#define KW_CASE(n) \
    case n: launch_pdl(k_colop_fanin<n>, nmap, 256, colop_park_bytes(job, reg_r1(n)), st, d_sims, d_t, map, nmap, job); break;
            KW_COLOP_SIZES(KW_CASE)
#undef KW_CASE
            default: break;
        }
        return;
    }
#define KW_CASE(NN, RR, MB)                                                                                 \
    if (n == NN && v.r1 == RR && v.minb == MB) {                                                            \
        launch_pdl(k_colop<NN, RR, MB>, nmap, 256, colop_park_bytes(job, RR), st, d_sims, d_t, map, nmap, job);     \
        return;                                                                                             \
    }
    KW_COLOP_VARIANTS(KW_CASE)
#undef KW_CASE
}

}  // namespace kw
