// kw_small.cu — the small kernels of a time step: t = 0 override, sources, sensor sampling,
// step counter, finiteness check, smoothing reductions and the intensity post-process.
#include "kw_device.cuh"

#include <algorithm>
#include <cstdlib>

namespace kw {

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
    if (S.psrc_q) return;   // precorrected: added by the density epilogue
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

// dst[idx[q]] = val[q] (setup: the scaled source mask of a precorrected pressure source)
__global__ void k_scatter(float* __restrict__ dst, const int* __restrict__ idx, const float* __restrict__ val, int n) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) dst[__ldg(idx + q)] = __ldg(val + q);
}

void launch_scatter(cudaStream_t st, float* dst, const int* idx, const float* val, int n) {
    if (n > 0) k_scatter<<<(n + 255) / 256, 256, 0, st>>>(dst, idx, val, n);
}

// sensor sampling + recording (Recording.swift:37-45, 129-168). which = 0: p, 1: velocity
// component `comp` (collocated field in tmp[comp]).
__device__ __forceinline__ void sample_one(const SimDev* __restrict__ sims, int t, int which, int comp) {
    const SimDev& S = sims[blockIdx.y];
    if (t >= S.nt) return;
    const SensorDev& sn = S.sensor;
    if (sn.kind == 0) return;
    if (which == 0 ? !(sn.record_p_series || sn.record_p_agg) : !(sn.record_u_series || sn.record_u_agg)) return;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= sn.npts) return;
    const float* f = which == 0 ? (sn.ndir > 0 ? sn.dir_field + (long long)__ldg(sn.dir_slot + q) * S.N : S.p) : S.tmp[comp];
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

// tick_count != null: this launch is the last of the step and also advances the step counter,
// once every CTA has read it (the last CTA to finish writes t + 1 and rearms the count)
__global__ void k_sample(const SimDev* __restrict__ sims, int* d_t, int which, int comp, unsigned int* tick_count) {
    pdl_enter();
    const int t = *d_t;
    sample_one(sims, t, which, comp);
    if (tick_count) {
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            if (atomicAdd(tick_count, 1u) == gridDim.x * gridDim.y - 1) {
                *tick_count = 0;
                *d_t = t + 1;
            }
        }
    }
}

__global__ void k_tick(int* d_t) {
    pdl_enter();
    *d_t += 1;
}

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
    // the pass kernels stage tiles of up to (opt-in limit - static shared memory) per CTA
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    init_r2c_attributes(optin);
    init_col_attributes(optin);
    init_c2r_attributes(optin);
    init_rowr_attributes(optin);
    init_colp_attributes();
    cudaFuncSetAttribute((const void*)k_intensity, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - 1024);
    cudaGetLastError();  // the attribute calls must not leave a sticky error behind
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

void launch_sample(cudaStream_t st, const SimDev* d_sims, int* d_t, int nsims, int max_pts, int which, int comp,
                   unsigned int* tick_count) {
    if (max_pts <= 0) return;
    dim3 g((max_pts + 255) / 256, nsims);
    launch_pdl(k_sample, g, 256, 0, st, d_sims, d_t, which, comp, tick_count);
}

void launch_tick(cudaStream_t st, int* d_t) { launch_pdl(k_tick, 1, 1, 0, st, d_t); }

// Opt-in (KW_PDL=1): on a B200 the 256^3 step, captured as a CUDA graph, took 1.67 ms with the
// attribute on every pass kernel against 1.46 ms without it (the per-launch times did not change).
bool pdl_enabled() {   // read on every launch (a test switches it between simulations)
    const char* e = std::getenv("KW_PDL");
    return e && e[0] == '1';
}

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
