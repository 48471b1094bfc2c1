// kw_adjoint.cu — pointwise and sparse kernels of the discrete adjoint of the time step
// (host orchestration in kw_adjoint.cpp; the spectral operators run through the ordinary pass
// kernels with FS_ADJ fields).
//
// Forward step t (kw_engine.cpp issue_step), per grid point, with d_a = D+_a p(t-1) for the
// velocity and d_a = D-_a u_a(t) for the density (D+-_a = Re F^-1(i k_a e^{+-i k_a dx_a/2} kappa F .)):
//   u_a   = sg_a (sg_a u_a - dtor_a D+_a p(t-1))
//   rho_a = pm_a (pm_a rho_a - dt rho0 nl d_a),   nl = (2 S(t-1) + rho0) / rho0 (B/A) or 1
//   rho_a += (1 / dx_a) G(src),  G = Re F^-1(cos(c_ref dt |k| / 2) F .),  src = sig 2 dt / (D c) at the mask
//   S = sum_a rho_a,  div = rho0 sum_a d_a
//   p = c^2 (S + tau A1(div) - eta A2(S) + B/A S^2 / (2 rho0))   (power law; Stokes: tau div)
// Reverse (lambda_x = dL/dx of the state after step t):
//   lambda_p += Sample^T r_t
//   dL/dc  += lambda_p (2 p / c + c ((y-1) tau A1(div) - y eta A2(S)))      (Stokes: + c tau div)
//             with tau A1(div) - eta A2(S) = p / c^2 - S - B/A S^2 / (2 rho0), so only A2(S) is needed:
//             the forward (recompute) step's dispersion epilogue keeps it on the tape
//   lE = c^2 lambda_p;  lS = lE + lE B/A S / rho0 - A2(eta lE);  ldiv = A1(tau lE) (Stokes: tau lE)
//   L_a = lambda_rho_a + lS;  source: dL/dc_i += G(sum_a L_a / dx_a)_i sig (-scale_i / c_i)
//   w_a = rho0 ldiv - pm_a dt rho0 nl L_a
//   lambda_rho_a <- pm_a^2 L_a - 2 dt sum_b pm_b d_b L_b   (the B/A term through nl)
//   mu_a = lambda_u_a - D+_a w_a                            ((D-_a)^T = -D+_a)
//   lambda_u_a <- sg_a^2 mu_a;  lambda_p <- sum_a D-_a(sg_a dtor_a mu_a)
#include "kw_adjoint.h"
#include "kw_device.cuh"

namespace kw {

__device__ __forceinline__ int layout_coord(const SimDev& S, long long i, int a) {
    const int L = a + 3 - S.dim;
    const long long ic = i % S.C;
    const long long r = i / S.C;
    const int ib = (int)(r % S.B);
    const int ia = (int)(r / S.B);
    return L == 0 ? ia : (L == 1 ? ib : (int)ic);
}

__global__ void k_set_step(int* d_t, int t) { *d_t = t; }

__device__ __forceinline__ void set_views(SimDev& S, const AdjTapeEntry& e) {
    S.adj[ADJ_PTP] = e.p;
    S.adj[ADJ_STP] = e.s;
    S.adj[ADJ_SPRP] = e.sprev;
    S.adj[ADJ_DIVP] = e.div;
    for (int b = 0; b < kMaxComp; ++b) S.adj[ADJ_DDP + b] = e.dd[b];
    S.adj[ADJ_Q2] = e.q2;
    S.adj[ADJ_PPREV] = e.pprev;
}

__global__ void k_adj_tape(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                           const AdjTapeEntry* __restrict__ table, int stokes) {
    const SimDev& S = sims[0];
    const int tn = *d_t;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.N) return;
    const AdjTapeEntry e = table[tn - 1];
    e.p[i] = S.p[i];
    e.s[i] = S.rho_sum[i];
    if (stokes) e.div[i] = S.div_term[i];
}

__global__ void k_adj_views(SimDev* __restrict__ sims, const AdjTapeEntry* __restrict__ table, int t) {
    set_views(sims[0], table[t]);
}

// Start of a reverse step: t = *d_rev (counted down by k_adj_eos); thread 0 sets the step counter
// *d_t = t and points the tape views at table[t]; every thread adds its sensor point's residual:
// lambda_p += Sample^T r_t (binary: one point; Cartesian: multilinear corners, which can coincide),
// and x1 = tau c^2 lambda_p, x2 = eta c^2 lambda_p at the same points.
__global__ void k_adj_begin(SimDev* __restrict__ sims, int* __restrict__ d_t, const int* __restrict__ d_rev,
                            const AdjTapeEntry* __restrict__ table, const float* __restrict__ resid) {
    SimDev& S = sims[0];
    const int t = *d_rev;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *d_t = t;
        set_views(S, table[t]);
    }
    const SensorDev& sn = S.sensor;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= sn.npts) return;
    const float r = resid[(long long)t * sn.npts + q];
    for (int c = 0; c < sn.ncorners; ++c) {
        const int i = __ldg(sn.idx + q * sn.ncorners + c);
        const float w = sn.kind == 2 ? __ldg(sn.w + q * sn.ncorners + c) : 1.f;
        const float v = w * r;
        atomicAdd(S.adj[ADJ_LP] + i, v);
        if (S.absorb >= 2) {
            const float c2 = S.c2.at(i);
            atomicAdd(S.adj[ADJ_X1] + i, S.tau.at(i) * c2 * v);
            if (S.absorb == 3) atomicAdd(S.adj[ADJ_X2] + i, S.eta.at(i) * c2 * v);
        }
    }
}

// Every input is loaded before the first store: the stores may alias the loads as far as the
// compiler knows, and interleaving them would serialise the loads. GRHO: also the direct terms of
// dL/drho0 (rho0 enters dt rho0 nl, the absorption input rho0 div, B/A S^2 / (2 rho0)).
template <bool GRHO>
__global__ void __launch_bounds__(256, 4) k_adj_eos(const SimDev* __restrict__ sims, AdjStepArgs A, int* __restrict__ d_rev) {
    const SimDev& S = sims[0];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *d_rev -= 1;   // every reader of this step's *d_rev (k_adj_begin) has finished
    if (i >= S.N) return;
    const int D = S.dim;
    const float c2 = S.c2.at(i), lp = A.lam_p[i], sv = S.adj[ADJ_STP][i], r0 = S.rho0.at(i), pv = S.adj[ADJ_PTP][i];
    float tau = 0.f, divp = 0.f, eta = 0.f, q2 = 0.f, bona = 0.f, a1 = 0.f, a2 = 0.f, spv = 0.f;
    if (S.absorb == 1) { tau = S.tau.at(i); divp = S.adj[ADJ_DIVP][i]; }
    if (S.absorb >= 2) a1 = A.a1[i];
    if (S.absorb == 3) { eta = S.eta.at(i); q2 = S.adj[ADJ_Q2][i]; a2 = A.a2[i]; }
    if (S.nonlinear) { bona = S.bona.at(i); spv = S.adj[ADJ_SPRP][i]; }
    float lr[kMaxComp], dd[kMaxComp], pm[kMaxComp];
#pragma unroll
    for (int a = 0; a < kMaxComp; ++a) {
        if (a >= D) break;
        lr[a] = A.lam_r[a][i];
        if (S.nonlinear || GRHO) dd[a] = S.adj[ADJ_DDP + a][i];
        pm[a] = __ldg(S.ax[a].pml + layout_coord(S, i, a));
    }
    double gcv = A.gc[i];
    const float c = sqrtf(c2);
    double dpdc = 2.0 * (double)pv / c;
    if (S.absorb == 1) dpdc += (double)c * tau * divp;
    if (S.absorb >= 2) {
        // (y-1) tau A1(div) - y eta A2(S) = (y-1) E - eta A2(S), E = tau A1(div) - eta A2(S) = p / c^2 - S - B/A S^2 / (2 rho0)
        double E = (double)pv / c2 - sv;
        if (S.nonlinear) E -= (double)bona * sv * sv / (2.0 * r0);
        double term = (double)(A.y - 1.f) * E;
        if (S.absorb == 3) term -= (double)eta * q2;
        dpdc += (double)c * term;
    }
    gcv += (double)lp * dpdc;
    const float lE = c2 * lp;
    float lS = lE;
    if (S.nonlinear) lS += lE * bona * sv / r0;
    if (S.absorb == 3) lS -= a2;
    float ldiv = 0.f;
    if (S.absorb == 1) ldiv = tau * lE;
    else if (S.absorb >= 2) ldiv = a1;
    const float nl = S.nonlinear ? (2.f * spv + r0) / r0 : 1.f;
    const float dtr = S.dt * r0;
    float lam[kMaxComp], w[kMaxComp];
    float lsprev = 0.f, sig = 0.f;
#pragma unroll
    for (int a = 0; a < kMaxComp; ++a) {
        if (a >= D) break;
        lam[a] = lr[a] + lS;
        w[a] = r0 * ldiv - pm[a] * dtr * nl * lam[a];
        if (S.nonlinear) lsprev += -2.f * S.dt * pm[a] * dd[a] * lam[a];
        sig += lam[a] * S.ax[a].inv_d;
    }
    A.gc[i] = gcv;
    if constexpr (GRHO) {
        // d p / d rho0 = c^2 (tau A1 or tau (Stokes)) sum_a d_a - c^2 B/A S^2 / (2 rho0^2);
        // d rho_a / d rho0 = -pm_a dt d_a (d(dt rho0 nl) / d rho0 = dt)
        float sd = 0.f;
        for (int a = 0; a < D; ++a) sd += dd[a];
        double g = 0.0;
        if (S.absorb >= 1) g += (double)ldiv * sd;
        if (S.nonlinear) g -= (double)lE * bona * sv * sv / (2.0 * (double)r0 * r0);
        for (int a = 0; a < D; ++a) g -= (double)pm[a] * S.dt * dd[a] * lam[a];
        S.adj_gr[i] += g;
    }
#pragma unroll
    for (int a = 0; a < kMaxComp; ++a) {
        if (a >= D) break;
        A.w[a][i] = w[a];
        A.lam_r[a][i] = pm[a] * pm[a] * lam[a] + lsprev;
    }
    if (A.sig) A.sig[i] = sig;
}

// dL/dc at the additive source points: G(sigma)_i sig (-scale_i / c_i)
__global__ void k_adj_src(const SimDev* __restrict__ sims, const float* __restrict__ gsig, const int* __restrict__ d_t,
                          double* __restrict__ gc) {
    const SimDev& S = sims[0];
    const int t = *d_t;
    const SourceDev& s = S.psrc;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= s.nsrc || t >= s.len) return;
    const float sg = __ldg(s.signal + (long long)(s.rows == 1 ? 0 : q) * s.len + t);
    const int i = __ldg(s.idx + q);
    const float c = sqrtf(S.c2.at(i));
    gc[i] += (double)gsig[i] * sg * (-(double)__ldg(s.scale[0] + q) / c);
}

// mu_a = lambda_u_a - e_a; lambda_u_a <- sg_a^2 mu_a; w_a <- sg_a dtor_a mu_a; with the density
// gradient also dL/d dtor_a += -sg_a g_a mu_a (g_a = D+_a p(t-1) in ADJ_GP)
__global__ void k_adj_vel(const SimDev* __restrict__ sims, AdjStepArgs A) {
    const SimDev& S = sims[0];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.N) return;
    for (int a = 0; a < S.dim; ++a) {
        const float mu = A.lam_u[a][i] - A.e[a][i];
        const float sg = __ldg(S.ax[a].pml_sg + layout_coord(S, i, a));
        if (S.adj_gr) S.adj_gdtor[a][i] -= (double)sg * S.adj[ADJ_GP + a][i] * mu;
        A.lam_u[a][i] = sg * sg * mu;
        A.w[a][i] = sg * S.dtor[a].at(i) * mu;
    }
}

// lambda_p = sum_a e_a and the next reverse step's absorption inputs (the fused form is the
// EPI_ADJ_SUM epilogue of the register row kernels)
__global__ void k_adj_sum(const SimDev* __restrict__ sims, AdjStepArgs A) {
    const SimDev& S = sims[0];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.N) return;
    float s = A.e[0][i];
    for (int a = 1; a < S.dim; ++a) s += A.e[a][i];
    A.lam_p[i] = s;
    if (S.absorb >= 2) {
        const float c2 = S.c2.at(i);
        S.adj[ADJ_X1][i] = S.tau.at(i) * c2 * s;
        if (S.absorb == 3) S.adj[ADJ_X2][i] = S.eta.at(i) * c2 * s;
    }
}

// the t = 0 override of an initial pressure: w_a = dtor_a / 2 lambda_u_a (then e_a = D-_a w_a)
__global__ void k_adj_half_dtor(const SimDev* __restrict__ sims, AdjStepArgs A) {
    const SimDev& S = sims[0];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.N) return;
    for (int a = 0; a < S.dim; ++a) A.w[a][i] = (S.dtor[a].at(i) / 2.f) * A.lam_u[a][i];
}

// dL/dp0 = lambda_p + sum_a lambda_rho_a / (D c^2) + sum_a (D+_a)^T(w_a) (= - e_a);
// dL/dc += sum_a lambda_rho_a p0 (-2 / (D c^3))
__global__ void k_adj_p0(const SimDev* __restrict__ sims, AdjStepArgs A, const float* __restrict__ p0s,
                         float* __restrict__ gp) {
    const SimDev& S = sims[0];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.N) return;
    const float c2 = S.c2.at(i);
    const float dd = S.dim == 1 ? 1.f : (float)S.dim;
    float lrs = 0.f, es = 0.f;
    for (int a = 0; a < S.dim; ++a) { lrs += A.lam_r[a][i]; es += A.e[a][i]; }
    if (gp) gp[i] = A.lam_p[i] + lrs / (dd * c2) - es;
    A.gc[i] += (double)lrs * p0s[i] * (-2.0 / ((double)dd * c2 * sqrtf(c2)));
}

__global__ void k_adj_store_grad(const double* __restrict__ gc, float* __restrict__ out, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (float)gc[i];
}

// t = 0 override u_a = dtor_a / 2 D+_a p0: dL/d dtor_a += lambda_u_a g_a / 2 (g_a in ADJ_GP)
__global__ void k_adj_rho_p0(const SimDev* __restrict__ sims) {
    const SimDev& S = sims[0];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.N) return;
    for (int a = 0; a < S.dim; ++a) S.adj_gdtor[a][i] += 0.5 * (double)S.adj[ADJ_LU + a][i] * S.adj[ADJ_GP + a][i];
}

// dL/drho0: the direct terms plus, per axis, staggerDensity^T (KSpaceFirstOrder.swift:799-806:
// rho_sg_a[i] = (rho0[i] + rho0[i + e_a]) / 2, the last index along a replicated) of
// dL/d rho_sg_a = dL/d dtor_a * d(dt / rho_sg) / d rho_sg = -dL/d dtor_a dtor_a^2 / dt
__global__ void k_adj_rho_final(const SimDev* __restrict__ sims, float* __restrict__ out) {
    const SimDev& S = sims[0];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.N) return;
    double g = S.adj_gr[i];
    for (int a = 0; a < S.dim; ++a) {
        const int L = a + 3 - S.dim;
        const long long stride = L == 0 ? (long long)S.B * S.C : (L == 1 ? (long long)S.C : 1LL);
        const int ia = layout_coord(S, i, a), n = S.ax[a].n;
        auto gsg = [&](long long j) {
            const double q = S.dtor[a].at(j);
            return -S.adj_gdtor[a][j] * q * q / (double)S.dt;
        };
        g += (ia == n - 1 ? 1.0 : 0.5) * gsg(i);   // rho_sg_a[i] holds rho0[i]
        if (ia >= 1) g += 0.5 * gsg(i - stride);    // rho_sg_a[i - e_a] holds rho0[i]
    }
    out[i] = (float)g;
}

// ---------------------------------------------------------------------------------------------
static unsigned blocks(long long n) { return (unsigned)((n + 255) / 256); }

void launch_set_step(cudaStream_t st, int* d_t, int t) { k_set_step<<<1, 1, 0, st>>>(d_t, t); }
void launch_adj_begin(cudaStream_t st, SimDev* d_sims, int* d_t, const int* d_rev, const AdjTapeEntry* table,
                      const float* resid, int npts) {
    k_adj_begin<<<blocks(npts > 0 ? npts : 1), 256, 0, st>>>(d_sims, d_t, d_rev, table, resid);
}
void launch_adj_tape(cudaStream_t st, SimDev* d_sims, const int* d_t, const AdjTapeEntry* table, int stokes, long long N) {
    k_adj_tape<<<blocks(N), 256, 0, st>>>(d_sims, d_t, table, stokes);
}
void launch_adj_views(cudaStream_t st, SimDev* d_sims, const AdjTapeEntry* table, int t) {
    k_adj_views<<<1, 1, 0, st>>>(d_sims, table, t);
}
void launch_adj_eos(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a, int* d_rev, bool grho) {
    if (grho) k_adj_eos<true><<<blocks(N), 256, 0, st>>>(d_sims, a, d_rev);
    else k_adj_eos<false><<<blocks(N), 256, 0, st>>>(d_sims, a, d_rev);
}
void launch_adj_src(cudaStream_t st, const SimDev* d_sims, int nsrc, const float* gsig, const int* d_t, double* gc) {
    if (nsrc > 0) k_adj_src<<<blocks(nsrc), 256, 0, st>>>(d_sims, gsig, d_t, gc);
}
void launch_adj_vel(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a) {
    k_adj_vel<<<blocks(N), 256, 0, st>>>(d_sims, a);
}
void launch_adj_sum(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a) {
    k_adj_sum<<<blocks(N), 256, 0, st>>>(d_sims, a);
}
void launch_adj_half_dtor(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a) {
    k_adj_half_dtor<<<blocks(N), 256, 0, st>>>(d_sims, a);
}
void launch_adj_p0(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a, const float* p0s, float* gp) {
    k_adj_p0<<<blocks(N), 256, 0, st>>>(d_sims, a, p0s, gp);
}
void launch_adj_store_grad(cudaStream_t st, const double* gc, float* out, long long n) {
    k_adj_store_grad<<<blocks(n), 256, 0, st>>>(gc, out, n);
}
void launch_adj_rho_p0(cudaStream_t st, const SimDev* d_sims, long long N) {
    k_adj_rho_p0<<<blocks(N), 256, 0, st>>>(d_sims);
}
void launch_adj_rho_final(cudaStream_t st, const SimDev* d_sims, long long N, float* out) {
    k_adj_rho_final<<<blocks(N), 256, 0, st>>>(d_sims, out);
}

}  // namespace kw
