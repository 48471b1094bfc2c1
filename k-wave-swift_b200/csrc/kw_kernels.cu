// kw_kernels.cu — sm_100a kernels of the k-space pseudospectral time step.
//
// A spectral operator application Re F^-1( H . F(x) ) on an [A][B][C] field runs as passes over
// HBM:
//   row pass   (C, contiguous):  R2C of real rows -> half-spectrum rows           k_row_r2c
//   column pass (B, then A):     C2C along the strided axes; the LAST forward pass also
//                                multiplies by H (and 1/N) and runs the inverse along the same
//                                axis while the tile is still in shared memory           k_col
//   row pass   (C):              C2R of half-spectrum rows with the physics update fused as an
//                                epilogue (velocity, density, EoS, source add, store)     k_row_c2r
// Every pass stages a tile of lines in shared memory, runs the Stockham FFT of kw_fft.cuh and
// writes the tile back with coalesced accesses. One launch covers the tiles of every simulation
// of an engine (BlockWork map), so a batch of small grids fills the GPU in one launch per pass.
#include "kw_fft.cuh"
#include "kw_kernels.cuh"

#include <cstdio>

namespace kw {

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
        default: return S.tmp[comp];
    }
}

__device__ __forceinline__ bool gate_open(const SimDev& S, int gate, int comp, int t) {
    if (t >= S.nt) return false;
    if (gate == GATE_PSRC) return S.has_p && t < S.psrc.len;
    if (gate == GATE_USRC) return S.has_u[comp] && t < S.usrc[comp].len;
    if (gate == GATE_P0) return S.has_p0 != 0;
    if (gate == GATE_ABS) return comp == 0 ? S.absorb >= 2 : S.absorb == 3;
    if (gate == GATE_RECU) return S.sensor.kind != 0 && (S.sensor.record_u_series || S.sensor.record_u_agg);
    return true;
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

// ------------------------------------------------------------------------------------------
// row pass: R2C
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_row_r2c(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                                 const BlockWork* __restrict__ map, RowR2CJob job) {
    extern __shared__ float2 sm[];
    __shared__ SimDev S;
    const BlockWork bw = map[blockIdx.x];
    load_sim(S, sims + bw.sim);
    const int t = *d_t;
    if (!gate_open(S, job.gate, bw.comp, t)) return;

    const int C = S.C, rows = S.A * S.B;
    const bool odd = (C & 1) != 0;
    const int M = odd ? C : C / 2;
    const int RPC = job.rows_per_cta;
    const int r0 = bw.tile * RPC;
    const int nl = min(RPC, rows - r0);
    const int ldi = RPC + 1;
    float2* bufA = sm;
    float2* bufB = sm + (size_t)M * ldi;
    const float* in = field_ptr(S, job.in_field, bw.comp) + (long long)r0 * C;

    for (int w = threadIdx.x; w < nl * M; w += blockDim.x) {
        const int l = w / M, m = w - l * M;
        float2 z;
        if (!odd) z = __ldg(reinterpret_cast<const float2*>(in + (long long)l * C) + m);
        else z = make_float2(__ldg(in + (long long)l * C + m), 0.f);
        bufA[m * ldi + l] = z;
    }
    __syncthreads();
    const float2* Z = fft_lines<false>(bufA, bufB, S.plan_row, nl, 1, ldi, true);

    float2* out = S.spec[job.spec_out + bw.comp] + (long long)r0 * S.Cp;
    const int Ch = S.Ch;
    const OpSpec op = job.op[bw.comp];
    for (int w = threadIdx.x; w < nl * Ch; w += blockDim.x) {
        const int l = w / Ch, k = w - l * Ch;
        float2 X;
        if (!odd) {
            const float2 zk = Z[(k == M ? 0 : k) * ldi + l];
            const float2 zm = Z[((M - k) % M) * ldi + l];
            const float2 E = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
            const float2 D = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y + zm.y));
            const float2 O = make_float2(D.y, -D.x);  // -i D
            X = cadd(E, cmul(O, __ldg(S.row_tw + k)));
        } else {
            X = Z[k * ldi + l];
        }
        if (job.apply_op) X = cmul(X, op_factor(S, op, 0, 0, k, (long long)(r0 + l) * S.Cp + k));
        out[(long long)l * S.Cp + k] = X;
    }
}

// ------------------------------------------------------------------------------------------
// column pass: C2C along layout axis A or B, optionally fused fwd -> operator -> inv
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_col(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                             const BlockWork* __restrict__ map, ColJob job) {
    extern __shared__ float2 sm[];
    __shared__ SimDev S;
    const BlockWork bw = map[blockIdx.x];
    load_sim(S, sims + bw.sim);
    const int t = *d_t;
    if (!gate_open(S, job.gate, bw.comp, t)) return;

    const bool axisA = job.layout_axis == 0;
    const int n = axisA ? S.A : S.B;
    const int inner = axisA ? S.B * S.Cp : S.Cp;
    const FFTPlanDev& pl = axisA ? S.plan_a : S.plan_b;
    const int TW = job.tw_cols;
    const int nchunks = (inner + TW - 1) / TW;
    const int o = bw.tile / nchunks;
    const int c0 = (bw.tile - o * nchunks) * TW;
    const int ncols = min(TW, inner - c0);
    float2* X0 = sm;
    float2* X1 = sm + (size_t)n * TW;
    float2* X2 = sm + (size_t)2 * n * TW;
    const long long obase = (long long)o * n * inner + c0;
    const int comp_in = job.fanout ? 0 : bw.comp;
    const float2* in = S.spec[job.spec_in + comp_in] + obase;

    for (int w = threadIdx.x; w < n * TW; w += blockDim.x) {
        const int i = w / TW, l = w - i * TW;
        X0[w] = l < ncols ? in[(long long)i * inner + l] : make_float2(0.f, 0.f);
    }
    __syncthreads();

    if (job.mode != COL_FWD_OP_INV) {
        const float2* R = job.mode == COL_FWD ? fft_lines<false>(X0, X1, pl, TW, 1, TW, true)
                                              : fft_lines<true>(X0, X1, pl, TW, 1, TW, true);
        float2* out = S.spec[job.spec_in + comp_in] + obase;
        for (int w = threadIdx.x; w < n * TW; w += blockDim.x) {
            const int i = w / TW, l = w - i * TW;
            if (l < ncols) out[(long long)i * inner + l] = R[w];
        }
        return;
    }

    float2* F = fft_lines<false>(X0, X1, pl, TW, 1, TW, true);
    float2* P = F == X0 ? X1 : X0;
    float2* Q = X2;
    const int nouts = job.fanout ? job.nout : 1;
    for (int oo = 0; oo < nouts; ++oo) {
        const int oc = job.fanout ? oo : bw.comp;
        const OpSpec op = job.op[oc];
        for (int w = threadIdx.x; w < n * TW; w += blockDim.x) {
            const int i = w / TW, l = w - i * TW;
            const int c = c0 + l;
            float2 v = make_float2(0.f, 0.f);
            if (l < ncols) {
                int ka, kb, kc;
                if (axisA) { ka = i; kb = c / S.Cp; kc = c - kb * S.Cp; }
                else { ka = o; kb = i; kc = c; }
                if (kc < S.Ch) v = cmul(F[w], op_factor(S, op, ka, kb, kc, ((long long)ka * S.B + kb) * S.Cp + kc));
            }
            P[w] = v;
        }
        __syncthreads();
        const float2* R = fft_lines<true>(P, Q, pl, TW, 1, TW, true);
        float2* out = S.spec[job.spec_out + oc] + obase;
        for (int w = threadIdx.x; w < n * TW; w += blockDim.x) {
            const int i = w / TW, l = w - i * TW;
            if (l < ncols) out[(long long)i * inner + l] = R[w];
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------------
// row pass: C2R + fused epilogue
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void epi_point(const SimDev& S, const RowC2RJob& job, int comp0, int ncomp, long long i,
                                          int ca, int cb, int cc, const float* d) {
    auto coord = [&](int ax) { const int L = ax + 3 - S.dim; return L == 0 ? ca : (L == 1 ? cb : cc); };
    switch (job.epi) {
        case EPI_STORE:
            for (int o = 0; o < ncomp; ++o) field_ptr(S, job.out_field, comp0 + o)[i] = d[o];
            break;
        case EPI_VEL:  // u = pml_sg (pml_sg u - dt/rho_sg dp)   (KSpaceFirstOrder.swift:453-454)
            for (int o = 0; o < ncomp; ++o) {
                const int a = comp0 + o;
                const float sg = __ldg(S.ax[a].pml_sg + coord(a));
                float* u = S.u[a];
                u[i] = sg * (sg * u[i] - S.dtor[a].at(i) * d[o]);
            }
            break;
        case EPI_VEL_INIT:  // u = (dt/rho_sg / 2) dp0   (KSpaceFirstOrder.swift:519-520)
            for (int o = 0; o < ncomp; ++o) {
                const int a = comp0 + o;
                S.u[a][i] = (S.dtor[a].at(i) / 2.f) * d[o];
            }
            break;
        case EPI_ADD_U:
            for (int o = 0; o < ncomp; ++o) S.u[comp0 + o][i] += d[o];
            break;
        case EPI_DEN: {  // KSpaceFirstOrder.swift:457-465 (+ EoS when pointwise)
            float nl = 1.f;
            if (S.nonlinear) {
                float rp = 0.f;
                for (int a = 0; a < S.dim; ++a) rp = a == 0 ? S.rho[0][i] : rp + S.rho[a][i];
                const float r0 = S.rho0.at(i);
                nl = (2.f * rp + r0) / r0;
            }
            const float dtr = S.dtrho0.at(i);
            float rs = 0.f, dv = 0.f;
            for (int a = 0; a < S.dim; ++a) {
                const float pm = __ldg(S.ax[a].pml + coord(a));
                const float mass = S.nonlinear ? dtr * d[a] * nl : dtr * d[a];
                const float r = pm * (pm * S.rho[a][i] - mass);
                S.rho[a][i] = r;
                rs = a == 0 ? r : rs + r;
                dv = a == 0 ? d[a] : dv + d[a];
            }
            S.rho_sum[i] = rs;
            float divterm = 0.f;
            if (S.absorb >= 1) {
                divterm = S.rho0.at(i) * dv;
                S.div_term[i] = divterm;
            }
            if (S.eos_pointwise) S.p[i] = eos_point(S, i, rs, divterm);
            break;
        }
        case EPI_ADD_RHO: {  // additive p source, k-space corrected (KSpaceFirstOrder.swift:167-172)
            float rs = 0.f;
            for (int a = 0; a < S.dim; ++a) {
                const float r = S.rho[a][i] + d[0] * S.ax[a].inv_d;
                S.rho[a][i] = r;
                rs = a == 0 ? r : rs + r;
            }
            S.rho_sum[i] = rs;
            if (S.eos_pointwise) S.p[i] = eos_point(S, i, rs, S.absorb == 1 ? S.div_term[i] : 0.f);
            break;
        }
        case EPI_EOS_ABS: {  // power-law absorption / dispersion (KSpaceFirstOrder.swift:836-845)
            const float rs = S.rho_sum[i];
            float term = S.tau.at(i) * d[0];
            if (S.absorb == 3) term = term - S.eta.at(i) * d[1];
            float e = rs + term;
            if (S.nonlinear) e = e + S.bona.at(i) * (rs * rs) / (2.f * S.rho0.at(i));
            S.p[i] = S.c2.at(i) * e;
            break;
        }
        default: break;
    }
}

__global__ void __launch_bounds__(256) k_row_c2r(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                                 const BlockWork* __restrict__ map, RowC2RJob job) {
    extern __shared__ float2 sm[];
    __shared__ SimDev S;
    const BlockWork bw = map[blockIdx.x];
    load_sim(S, sims + bw.sim);
    const int t = *d_t;
    if (!gate_open(S, job.gate, bw.comp, t)) return;

    const int C = S.C, rows = S.A * S.B;
    const bool odd = (C & 1) != 0;
    const int M = odd ? C : C / 2;
    const int RPC = job.rows_per_cta;
    const int r0 = bw.tile * RPC;
    const int nl = min(RPC, rows - r0);
    const int ncomp = job.ncomp;
    const int comp0 = ncomp == 1 ? bw.comp : 0;
    const int lines = nl * ncomp;
    const int ldi = RPC * ncomp + 1;
    float2* bufA = sm;
    float2* bufB = sm + (size_t)M * ldi;

    for (int w = threadIdx.x; w < lines * M; w += blockDim.x) {
        const int line = w / M, k = w - line * M;
        const int cc = line / nl, l = line - cc * nl;
        const float2* X = S.spec[job.spec_in + comp0 + cc] + (long long)(r0 + l) * S.Cp;
        float2 z;
        if (!odd) {
            float2 a = X[k], b = X[M - k];
            if (k == 0) { a.y = 0.f; b.y = 0.f; }          // self-conjugate bins: real part only
            const float2 s = make_float2(a.x + b.x, a.y - b.y);    // a + conj(b)
            const float2 dd = make_float2(a.x - b.x, a.y + b.y);   // a - conj(b)
            const float2 e = cmulc(dd, __ldg(S.row_tw + k));       // dd * exp(+2 pi i k / C)
            z = make_float2(s.x - e.y, s.y + e.x);                 // s + i e
        } else {
            if (k < S.Ch) z = X[k];
            else { const float2 v = X[C - k]; z = make_float2(v.x, -v.y); }
            if (k == 0) z.y = 0.f;
        }
        bufA[k * ldi + line] = z;
    }
    __syncthreads();
    const float2* Z = fft_lines<true>(bufA, bufB, S.plan_row, lines, 1, ldi, true);

    const int B = S.B;
    for (int w = threadIdx.x; w < nl * M; w += blockDim.x) {
        const int l = w / M, m = w - l * M;
        const int row = r0 + l;
        const int ca = row / B, cb = row - ca * B;
        float d0[kMaxComp], d1[kMaxComp];
        for (int cc = 0; cc < ncomp; ++cc) {
            const float2 z = Z[m * ldi + cc * nl + l];
            d0[cc] = z.x;
            d1[cc] = z.y;
        }
        if (!odd) {
            const long long i0 = (long long)row * C + 2 * m;
            epi_point(S, job, comp0, ncomp, i0, ca, cb, 2 * m, d0);
            epi_point(S, job, comp0, ncomp, i0 + 1, ca, cb, 2 * m + 1, d1);
        } else {
            epi_point(S, job, comp0, ncomp, (long long)row * C + m, ca, cb, m, d0);
        }
    }
}

// ------------------------------------------------------------------------------------------
// small kernels
// ------------------------------------------------------------------------------------------

// t = 0 override for an initial pressure: p = p0, rho_a = p0 / (d c^2) (1D: p0 / c^2)
// (KSpaceFirstOrder.swift:514-517, 1D :322-323). The velocity part runs as a spectral job.
__global__ void k_init_p0(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                          const BlockWork* __restrict__ map, const float* const* __restrict__ p0s) {
    __shared__ SimDev S;
    const BlockWork bw = map[blockIdx.x];
    load_sim(S, sims + bw.sim);
    const float* p0 = p0s[bw.sim];
    if (!p0) return;
    const long long i = (long long)bw.tile * blockDim.x + threadIdx.x;
    if (i >= S.N) return;
    const float f = p0[i];
    S.p[i] = f;
    const float c2 = S.c2.at(i);
    const float r = S.dim == 1 ? f / c2 : f / ((float)S.dim * c2);
    float rs = 0.f;
    for (int a = 0; a < S.dim; ++a) {
        S.rho[a][i] = r;
        rs = a == 0 ? r : rs + r;
    }
    S.rho_sum[i] = rs;
}

__device__ __forceinline__ float src_value(const SourceDev& s, int q, int t) {
    return __ldg(s.signal + (size_t)(s.rows == 1 ? 0 : q) * s.len + t);
}

// velocity sources (KSpaceFirstOrder.swift:497-501): dirichlet / additive-no-correction act on u
// directly; additive scatters the scaled values into the sparse source field.
__global__ void k_src_u(const SimDev* __restrict__ sims, const int* __restrict__ d_t, int scatter_only) {
    const SimDev& S = sims[blockIdx.y];
    const int t = *d_t;
    if (t >= S.nt) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    for (int a = 0; a < S.dim; ++a) {
        if (!S.has_u[a]) continue;
        const SourceDev& s = S.usrc[a];
        if (q >= s.nsrc || t >= s.len) continue;
        const bool additive = s.mode == 1;
        if (additive != (scatter_only != 0)) continue;
        const float v = src_value(s, q, t) * __ldg(s.scale[0] + q);
        const int i = __ldg(s.idx + q);
        if (s.mode == 0) S.u[a][i] = v;
        else if (s.mode == 2) S.u[a][i] += v;
        else S.src_buf[a][i] = v;
    }
}

// pressure sources (KSpaceFirstOrder.swift:503-508), applied to every split density rho_a.
__global__ void k_src_p(const SimDev* __restrict__ sims, const int* __restrict__ d_t, int scatter_only) {
    const SimDev& S = sims[blockIdx.y];
    const int t = *d_t;
    if (t >= S.nt || !S.has_p) return;
    const SourceDev& s = S.psrc;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= s.nsrc || t >= s.len) return;
    const bool additive = s.mode == 1;
    if (additive != (scatter_only != 0)) return;
    const float sig = src_value(s, q, t);
    const int i = __ldg(s.idx + q);
    if (additive) {
        S.src_buf[0][i] = sig * __ldg(s.scale[0] + q);
        return;
    }
    float rs = 0.f;
    for (int a = 0; a < S.dim; ++a) {
        float r;
        if (s.mode == 0) r = sig * __ldg(s.scale[0] + q);
        else r = S.rho[a][i] + sig * __ldg(s.scale[a] + q);
        S.rho[a][i] = r;
        rs = a == 0 ? r : rs + r;
    }
    S.rho_sum[i] = rs;
    if (S.eos_pointwise) S.p[i] = eos_point(S, i, rs, S.absorb == 1 ? S.div_term[i] : 0.f);
}

// sensor sampling + recording (Recording.swift:37-45, 129-168). which = 0: p, 1: velocity
// component `comp` (collocated field in tmp[comp]).
__global__ void k_sample(const SimDev* __restrict__ sims, const int* __restrict__ d_t, int which, int comp) {
    const SimDev& S = sims[blockIdx.y];
    const int t = *d_t;
    if (t >= S.nt) return;
    const SensorDev& sn = S.sensor;
    if (sn.kind == 0) return;
    if (which == 0 ? !(sn.record_p_series || sn.record_p_agg) : !(sn.record_u_series || sn.record_u_agg)) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= sn.npts) return;
    const float* f = which == 0 ? S.p : S.tmp[comp];
    float v;
    if (sn.kind == 1) {
        v = f[__ldg(sn.idx + q)];
    } else {
        v = 0.f;
        for (int c = 0; c < sn.ncorners; ++c)
            v = c == 0 ? f[__ldg(sn.idx + q * sn.ncorners)] * __ldg(sn.w + q * sn.ncorners)
                       : v + f[__ldg(sn.idx + q * sn.ncorners + c)] * __ldg(sn.w + q * sn.ncorners + c);
    }
    if (!isfinite(v)) atomicOr(S.nonfinite, 1);
    if (which == 0) {
        if (sn.record_p_series) sn.p_series[(long long)t * sn.npts + q] = v;
        if (sn.record_p_agg) {
            sn.p_max[q] = t == 0 ? v : fmaxf(sn.p_max[q], v);
            sn.p_min[q] = t == 0 ? v : fminf(sn.p_min[q], v);
            // Kahan-compensated running sum of p^2
            const float s = t == 0 ? 0.f : sn.p_ss[q];
            const float c = t == 0 ? 0.f : sn.p_ssc[q];
            const float y = v * v - c;
            const float tt = s + y;
            sn.p_ssc[q] = (tt - s) - y;
            sn.p_ss[q] = tt;
        }
    } else {
        if (sn.record_u_series) sn.u_series[comp][(long long)t * sn.npts + q] = v;
        if (sn.record_u_agg) {
            sn.u_max[comp][q] = t == 0 ? v : fmaxf(sn.u_max[comp][q], v);
            const float s = t == 0 ? 0.f : sn.u_ss[comp][q];
            const float c = t == 0 ? 0.f : sn.u_ssc[comp][q];
            const float y = v * v - c;
            const float tt = s + y;
            sn.u_ssc[comp][q] = (tt - s) - y;
            sn.u_ss[comp][q] = tt;
        }
    }
}

__global__ void k_tick(int* d_t) { *d_t += 1; }

__global__ void k_check_finite(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                               const BlockWork* __restrict__ map) {
    const BlockWork bw = map[blockIdx.x];
    const SimDev& S = sims[bw.sim];
    const long long i = (long long)bw.tile * blockDim.x + threadIdx.x;
    if (i >= S.N) return;
    if (!isfinite(S.p[i])) atomicOr(S.nonfinite, 1);
}

__global__ void k_absmax(const float* __restrict__ x, long long n, unsigned int* out) {
    float m = 0.f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(x[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// x *= num / den when den > 0 (smooth(..., restore_max), Filters.swift:343-346)
__global__ void k_scale(float* x, long long n, const unsigned int* num, const unsigned int* den) {
    const float a = __uint_as_float(*num), b = __uint_as_float(*den);
    const float s = b > 0.f ? a / b : 1.f;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = x[i] * s;
}

// time-averaged intensity of one sensor point per block (Recording.swift:113-124):
// mean_t p[t] * sum_t' u[t'] h[(t - t') mod T], h = Re ifft(exp(i w / 2)) precomputed in FP64.
__global__ void k_intensity(const float* __restrict__ p, const float* __restrict__ u, int T, int npts,
                            const float* __restrict__ h, float* __restrict__ out) {
    extern __shared__ float su[];
    __shared__ double red[32];
    const int q = blockIdx.x;
    for (int t = threadIdx.x; t < T; t += blockDim.x) su[t] = u[(long long)t * npts + q];
    __syncthreads();
    double acc = 0.0;
    for (int t = threadIdx.x; t < T; t += blockDim.x) {
        double us = 0.0;
        for (int tp = 0; tp < T; ++tp) {
            int m = t - tp;
            m += m < 0 ? T : 0;
            us += (double)su[tp] * (double)__ldg(h + m);
        }
        acc += (double)p[(long long)t * npts + q] * us;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        out[q] = (float)(s / T);
    }
}

// ------------------------------------------------------------------------------------------
// host launchers
// ------------------------------------------------------------------------------------------
void init_kernel_attributes() {
    // The pass kernels stage tiles of up to (opt-in limit - static shared memory) per CTA.
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const void* fns[] = {(const void*)k_row_r2c, (const void*)k_col, (const void*)k_row_c2r, (const void*)k_intensity};
    for (const void* fn : fns) {
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess) continue;
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    }
    cudaGetLastError();  // the attribute calls must not leave a sticky error behind
}

void launch_row_r2c(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nblocks,
                    const RowR2CJob& job, size_t smem) {
    if (nblocks <= 0) return;
    k_row_r2c<<<nblocks, 256, smem, st>>>(d_sims, d_t, map, job);
}

void launch_col(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nblocks,
                const ColJob& job, size_t smem) {
    if (nblocks <= 0) return;
    k_col<<<nblocks, 256, smem, st>>>(d_sims, d_t, map, job);
}

void launch_row_c2r(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nblocks,
                    const RowC2RJob& job, size_t smem) {
    if (nblocks <= 0) return;
    k_row_c2r<<<nblocks, 256, smem, st>>>(d_sims, d_t, map, job);
}

void launch_init_p0(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nblocks,
                    const float* const* d_p0s) {
    if (nblocks <= 0) return;
    k_init_p0<<<nblocks, 256, 0, st>>>(d_sims, d_t, map, d_p0s);
}

void launch_src_u(cudaStream_t st, const SimDev* d_sims, const int* d_t, int nsims, int max_src, int scatter_only) {
    if (max_src <= 0) return;
    dim3 g((max_src + 255) / 256, nsims);
    k_src_u<<<g, 256, 0, st>>>(d_sims, d_t, scatter_only);
}

void launch_src_p(cudaStream_t st, const SimDev* d_sims, const int* d_t, int nsims, int max_src, int scatter_only) {
    if (max_src <= 0) return;
    dim3 g((max_src + 255) / 256, nsims);
    k_src_p<<<g, 256, 0, st>>>(d_sims, d_t, scatter_only);
}

void launch_sample(cudaStream_t st, const SimDev* d_sims, const int* d_t, int nsims, int max_pts, int which,
                   int comp) {
    if (max_pts <= 0) return;
    dim3 g((max_pts + 255) / 256, nsims);
    k_sample<<<g, 256, 0, st>>>(d_sims, d_t, which, comp);
}

void launch_tick(cudaStream_t st, int* d_t) { k_tick<<<1, 1, 0, st>>>(d_t); }

void launch_check_finite(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nblocks) {
    if (nblocks <= 0) return;
    k_check_finite<<<nblocks, 256, 0, st>>>(d_sims, d_t, map);
}

void launch_absmax(cudaStream_t st, const float* x, long long n, unsigned int* d_out_bits) {
    int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 8);
    if (blocks < 1) blocks = 1;
    k_absmax<<<blocks, 256, 0, st>>>(x, n, d_out_bits);
}

void launch_scale(cudaStream_t st, float* x, long long n, const unsigned int* d_num_bits, const unsigned int* d_den_bits) {
    int blocks = (int)std::min<long long>((n + 255) / 256, 148 * 8);
    if (blocks < 1) blocks = 1;
    k_scale<<<blocks, 256, 0, st>>>(x, n, d_num_bits, d_den_bits);
}

void launch_intensity(cudaStream_t st, const float* p_series, const float* u_series, int nt_used, int npts,
                      const float* h, float* out) {
    if (npts <= 0 || nt_used <= 0) return;
    size_t smem = (size_t)nt_used * sizeof(float);
    k_intensity<<<npts, 256, smem, st>>>(p_series, u_series, nt_used, npts, h, out);
}

}  // namespace kw
