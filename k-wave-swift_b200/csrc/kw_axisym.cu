// kw_axisym.cu — pointwise kernels of the axisymmetric solver (kspaceFirstOrderAS,
// Solver/KSpaceFirstOrderAS.swift:19-309). The grid is [nx][ny] with x axial and y radial (r >= 0);
// its spectral operators act on the 4x radial expansion [nx][4 ny] of each field, mirrored with the
// field's symmetry, and run through the ordinary pass kernels on a second simulation descriptor
// that describes the expanded grid (kw_axisym.cpp). These kernels mirror fields into that grid,
// take the trimmed results back (columns j < ny) and apply the axisymmetric updates:
//   ux = pml_x,sg (pml_x,sg ux - dt/rho_sg,x dp/dx),  uy = pml_y,sg (pml_y,sg uy - dt/rho_sg,y dp/dy)
//   rho_x = pml_x (pml_x rho_x - dt rho0 nl dux/dx),  rho_y = pml_y (pml_y rho_y - dt rho0 nl duy/dy)
//   p = c^2 (rho_x + rho_y + tau rho0 (dux/dx + duy/dy) + B/A (rho_x + rho_y)^2 / (2 rho0))
// with duy/dy carrying the cylindrical uy / r term, nl = (2 (rho_x + rho_y) + rho0) / rho0 with
// B/A; the radial PML acts at the outer edge only (its profiles are set up that way).
#include "../../include/kwave_cuda.h"
#include "kw_device.cuh"
#include "kw_kernels.cuh"

namespace kw {

namespace {

__device__ __forceinline__ float fld(const FieldOrScalar& f, long long i) { return f.ptr ? f.ptr[i] : f.s; }

// expanded column j of mirror `kind` -> (source column, sign); src = -1 for the WSWA zero columns
__device__ __forceinline__ int mirror_src(int kind, int ny, int j, float& sg) {
    const int q = j / ny, r = j - q * ny;
    if (kind == AS_WSWA) {   // [w, 0, -w(ny-1..1), -w, 0, w(ny-1..1)]
        if (q == 0) { sg = 1.f; return r; }
        if (q == 2) { sg = -1.f; return r; }
        if (r == 0) { sg = 0.f; return -1; }
        sg = q == 1 ? -1.f : 1.f;
        return ny - r;
    }
    // HAHS: [w, flip w, -w, -flip w]; HSHA: [w, -flip w, -w, flip w]
    const bool flip = q == 1 || q == 3;
    float s = q >= 2 ? -1.f : 1.f;
    if (kind == AS_HSHA && flip) s = -s;
    sg = s;
    return flip ? ny - 1 - r : r;
}

__global__ void k_as_mirror(const SimDev* __restrict__ std_sim, const SimDev* __restrict__ car, const float* __restrict__ src,
                            float* __restrict__ dst, int kind, int over_r) {
    const SimDev& S = *std_sim;
    const int nx = S.B, ny = S.C, nye = car->C;
    const long long n = (long long)nx * nye;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int i = (int)(e / nye), j = (int)(e - (long long)i * nye);
    float sg;
    const int r = mirror_src(kind, ny, j, sg);
    float v = 0.f;
    if (r >= 0) {
        v = src[(long long)i * ny + r];
        if (over_r) v *= S.ax[1].inv_d / (r + 0.5f);   // 1 / r on the staggered radial grid
    }
    dst[e] = sg * v;
}

// velocity update from the trimmed gradients g0 = dp/dx, g1 = dp/dy (expanded rows); with
// `init` the t = 0 override u_a = dt/rho_sg,a / 2 dp/da
__global__ void k_as_vel(const SimDev* __restrict__ std_sim, const float* __restrict__ g0, const float* __restrict__ g1,
                         int nye, int init) {
    const SimDev& S = *std_sim;
    const int nx = S.B, ny = S.C;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nx * ny) return;
    const int x = (int)(i / ny), y = (int)(i - (long long)x * ny);
    const long long e = (long long)x * nye + y;
    const float dx = g0[e], dy = g1[e];
    const float rx = fld(S.dtor[0], i), ry = fld(S.dtor[1], i);
    if (init) {
        S.u[0][i] = rx / 2.f * dx;
        S.u[1][i] = ry / 2.f * dy;
        return;
    }
    const float px = S.ax[0].pml_sg[x], py = S.ax[1].pml_sg[y];
    S.u[0][i] = px * (px * S.u[0][i] - rx * dx);
    S.u[1][i] = py * (py * S.u[1][i] - ry * dy);
}

// density update from dux/dx = d0 and duy/dy = d1 + d2 (expanded rows); keeps the divergence
__global__ void k_as_den(const SimDev* __restrict__ std_sim, const float* __restrict__ d0, const float* __restrict__ d1,
                         const float* __restrict__ d2, int nye) {
    const SimDev& S = *std_sim;
    const int nx = S.B, ny = S.C;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nx * ny) return;
    const int x = (int)(i / ny), y = (int)(i - (long long)x * ny);
    const long long e = (long long)x * nye + y;
    const float dux = d0[e], duy = d1[e] + d2[e];
    const float r0 = fld(S.rho0, i);
    float rx = S.rho[0][i], ry = S.rho[1][i];
    const float dtr = S.nonlinear ? S.dt * (2.f * (rx + ry) + r0) : S.dt * r0;
    const float pxv = S.ax[0].pml[x], pyv = S.ax[1].pml[y];
    rx = pxv * (pxv * rx - dtr * dux);
    ry = pyv * (pyv * ry - dtr * duy);
    S.rho[0][i] = rx;
    S.rho[1][i] = ry;
    S.div_term[i] = dux + duy;
}

// equation of state (Stokes absorption and B/A as the reference)
__global__ void k_as_eos(const SimDev* __restrict__ std_sim) {
    const SimDev& S = *std_sim;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.N) return;
    const float rt = S.rho[0][i] + S.rho[1][i];
    const float r0 = fld(S.rho0, i);
    float e = rt;
    if (S.absorb == 1) e = e + fld(S.tau, i) * r0 * S.div_term[i];
    if (S.nonlinear) e = e + fld(S.bona, i) * (rt * rt) / (2.f * r0);
    S.p[i] = fld(S.c2, i) * e;
    S.rho_sum[i] = rt;
}

// t = 0 override: p = p0, rho_x = rho_y = p0 / (2 c^2)
__global__ void k_as_p0(const SimDev* __restrict__ std_sim, const float* __restrict__ p0) {
    const SimDev& S = *std_sim;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.N) return;
    const float v = p0[i];
    S.p[i] = v;
    const float r = v / (2.f * fld(S.c2, i));
    S.rho[0][i] = r;
    S.rho[1][i] = r;
}

// Source values at step t (ScaledSource of KSpaceFirstOrderAS.swift:122-149). target 0: pressure
// (both density splits; Dirichlet sets, additive-no-correction adds, additive writes the scaled
// value divided by dx into the sparse field `buf`, zeros once the signal has ended); target 1, 2:
// ux, uy (Dirichlet sets, additive-no-correction adds, additive writes into `buf`).
__global__ void k_as_src(const SimDev* __restrict__ std_sim, const int* __restrict__ d_t, int target, float* __restrict__ buf) {
    const SimDev& S = *std_sim;
    const SourceDev& s = target == 0 ? S.psrc : S.usrc[target - 1];
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= s.nsrc) return;
    const int t = *d_t;
    const int i = __ldg(s.idx + q);
    const bool on = t < s.len && t < S.nt;
    if (s.mode == KW_SOURCE_ADDITIVE) {
        float v = 0.f;
        if (on) {
            v = __ldg(s.signal + (size_t)(s.rows == 1 ? 0 : q) * s.len + t) * __ldg(s.scale[0] + q);
            if (target == 0) v *= S.ax[0].inv_d;
        }
        buf[i] = v;
        return;
    }
    if (!on) return;
    const float v = __ldg(s.signal + (size_t)(s.rows == 1 ? 0 : q) * s.len + t) * __ldg(s.scale[0] + q);
    if (target == 0) {
        if (s.mode == KW_SOURCE_DIRICHLET) { S.rho[0][i] = v; S.rho[1][i] = v; }
        else { S.rho[0][i] += v; S.rho[1][i] += v; }
    } else {
        float* u = S.u[target - 1];
        if (s.mode == KW_SOURCE_DIRICHLET) u[i] = v;
        else u[i] += v;
    }
}

// add the trimmed expanded field `g` to f0 (and f1)
__global__ void k_as_add(const SimDev* __restrict__ std_sim, const float* __restrict__ g, int nye, float* __restrict__ f0,
                         float* __restrict__ f1) {
    const SimDev& S = *std_sim;
    const int nx = S.B, ny = S.C;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)nx * ny) return;
    const int x = (int)(i / ny), y = (int)(i - (long long)x * ny);
    const float v = g[(long long)x * nye + y];
    f0[i] += v;
    if (f1) f1[i] += v;
}

inline int blocks_of(long long n) { return (int)((n + 255) / 256); }

}  // namespace

void launch_as_mirror(cudaStream_t st, const SimDev* std_sim, const SimDev* car, long long n_exp, const float* src,
                      float* dst, int kind, int over_r) {
    k_as_mirror<<<blocks_of(n_exp), 256, 0, st>>>(std_sim, car, src, dst, kind, over_r);
}
void launch_as_vel(cudaStream_t st, const SimDev* std_sim, long long n, const float* g0, const float* g1, int nye, int init) {
    k_as_vel<<<blocks_of(n), 256, 0, st>>>(std_sim, g0, g1, nye, init);
}
void launch_as_den(cudaStream_t st, const SimDev* std_sim, long long n, const float* d0, const float* d1, const float* d2,
                   int nye) {
    k_as_den<<<blocks_of(n), 256, 0, st>>>(std_sim, d0, d1, d2, nye);
}
void launch_as_eos(cudaStream_t st, const SimDev* std_sim, long long n) { k_as_eos<<<blocks_of(n), 256, 0, st>>>(std_sim); }
void launch_as_p0(cudaStream_t st, const SimDev* std_sim, long long n, const float* p0) {
    k_as_p0<<<blocks_of(n), 256, 0, st>>>(std_sim, p0);
}
void launch_as_src(cudaStream_t st, const SimDev* std_sim, const int* d_t, int nsrc, int target, float* buf) {
    if (nsrc > 0) k_as_src<<<blocks_of(nsrc), 256, 0, st>>>(std_sim, d_t, target, buf);
}
void launch_as_add(cudaStream_t st, const SimDev* std_sim, long long n, const float* g, int nye, float* f0, float* f1) {
    k_as_add<<<blocks_of(n), 256, 0, st>>>(std_sim, g, nye, f0, f1);
}

}  // namespace kw
