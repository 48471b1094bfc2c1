// kw_device.cuh — device helpers shared by the pass kernels and the small kernels.
#pragma once

#include "kw_fft.cuh"
#include "kw_kernels.cuh"

namespace kw {

// ------------------------------------------------------------------------------------------
// Programmatic dependent launch of the step's kernels. A kernel started by launch_pdl may be
// scheduled while its predecessor grid drains: its first instruction waits until every
// prerequisite grid has completed and its memory is visible (griddepcontrol.wait), and then
// lets its own successor be scheduled (griddepcontrol.launch_dependents). Every kernel that
// launch_pdl starts calls pdl_enter() before anything else, so each one still runs after the
// whole of the previous one; for a launch without the attribute both are no-ops.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
bool pdl_enabled();   // KW_PDL=1 (kw_small.cu); off by default: plain stream order
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

// ------------------------------------------------------------------------------------------
// helpers
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void load_sim(SimDev& dst, const SimDev* __restrict__ src) {
    static_assert(sizeof(SimDev) % 4 == 0, "SimDev must be word sized");
    const int* s = reinterpret_cast<const int*>(src);
    int* d = reinterpret_cast<int*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(SimDev) / 4); i += blockDim.x) d[i] = __ldg(s + i);
    __syncthreads();
}

__device__ __forceinline__ float* field_ptr(const SimDev& S, int sel, int comp) {
    switch (sel) {
        case FS_P: return S.p;
        case FS_U: return S.u[comp];
        case FS_RHO: return S.rho[comp];
        case FS_RHO_SUM: return S.rho_sum;
        case FS_DIV: return S.div_term;
        case FS_SRCBUF: return S.src_buf[comp];
        case FS_WORK: return comp == 0 ? S.div_term : S.rho_sum;   // power-law inputs
        case FS_TMP: return S.tmp[comp];
        default:
            if (sel >= FS_DIR) return S.sensor.dir_field + (long long)(sel - FS_DIR + comp) * S.N;
            return S.adj[sel - FS_ADJ + comp];
    }
}

__device__ __forceinline__ bool gate_open(const SimDev& S, int gate, int comp, int t) {
    if (t >= S.nt) return false;
    if (gate == GATE_PSRC) return S.has_p && !S.psrc_q && t < S.psrc.len;
    if (gate == GATE_USRC) return S.has_u[comp] && t < S.usrc[comp].len;
    if (gate == GATE_P0) return S.has_p0 != 0;
    if (gate == GATE_ABS) return comp == 0 ? S.absorb >= 2 : S.absorb == 3;
    if (gate == GATE_RECU) return S.sensor.kind != 0 && (S.sensor.record_u_series || S.sensor.record_u_agg);
    if (gate >= GATE_DIR) return gate - GATE_DIR < S.sensor.ndir;
    return true;
}

// Signal value at step t of a simulation's precorrected additive pressure source (SimDev::psrc_q);
// 0 once the signal has ended or when the simulation has none.
__device__ __forceinline__ float psrc_gain(const SimDev& S, int t) {
    return (S.psrc_q && S.has_p && t < S.psrc.len) ? __ldg(S.psrc.signal + t) : 0.f;
}

// wavenumber index along reference axis `ax` for spectrum coordinates (ka, kb, kc)
__device__ __forceinline__ int axis_index(const SimDev& S, int ax, int ka, int kb, int kc) {
    const int L = ax + 3 - S.dim;
    return L == 0 ? ka : (L == 1 ? kb : kc);
}

__device__ __forceinline__ float2 op_factor(const SimDev& S, const OpSpec& op, int ka, int kb, int kc, long long flat) {
    float2 f = make_float2(S.inv_n, 0.f);
    if (op.axis_op != AO_NONE) {
        const AxisDev& ax = S.ax[op.axis];
        const int idx = axis_index(S, op.axis, ka, kb, kc);
        const float2* v = op.axis_op == AO_DPOS ? ax.dpos : (op.axis_op == AO_DNEG ? ax.dneg : ax.colloc);
        f = cscale(__ldg(v + idx), S.inv_n);
    }
    if (op.radial != RT_NONE) f = cscale(f, __ldg(S.radial[op.radial] + flat));
    return f;
}

// equation of state at one point when it is pointwise (lossless / Stokes / B/A):
// p = c0^2 (rho + tau rho0 divU + B/A rho^2 / (2 rho0))   (KSpaceFirstOrder.swift:467-474, 836-845, 897)
__device__ __forceinline__ float eos_point(const SimDev& S, long long i, float rs, float divterm) {
    float e = rs;
    if (S.absorb == 1) e = e + S.tau.at(i) * divterm;
    if (S.nonlinear) e = e + S.bona.at(i) * (rs * rs) / (2.f * S.rho0.at(i));
    return S.c2.at(i) * e;
}


}  // namespace kw
