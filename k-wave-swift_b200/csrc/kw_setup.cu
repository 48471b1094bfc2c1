// kw_setup.cu — once-per-simulation setup computed on the device in FP64 (rounded to FP32 at the
// end, as the host-side FP64 restatement it replaces): the medium-derived fields and the radial
// (|k|-only) operator tables. The host uploads only the caller's FP32 c0 / rho0 / alpha maps and
// the per-axis FP64 wavenumber vectors, instead of computing and copying every derived field.
//
//   c2 = c0^2                                                     (KSpaceFirstOrder.swift:399)
//   dt / rho_sg_a, rho_sg_a = staggerDensity(rho0, a)             (KSpaceFirstOrder.swift:401-402, 799-806)
//   tau = -2 alpha_Np c0^(y-1), eta = 2 alpha_Np c0^y tan(pi y/2) (power law, KSpaceFirstOrder.swift:851-882)
//   tau = -2 alpha_Np c0                                          (Stokes)
//   kappa = sinc(c_ref dt |k| / 2), cos(c_ref dt |k| / 2), |k|^(y-2), |k|^(y-1) (0 at k = 0)
//                                                                 (KSpaceFirstOrder.swift:376-378, 812-826)
#include "kw_kernels.cuh"

#include <algorithm>
#include <cstring>

namespace kw {

__global__ void k_setup_c2(const float* __restrict__ c0, float* __restrict__ c2, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double c = c0[i];
        c2[i] = (float)(c * c);
    }
}

// dt / rho_sg along the layout axis with `stride` and length `len` (mean of neighbours, the last
// index replicated)
__global__ void k_setup_dtor(const float* __restrict__ rho0, float* __restrict__ out, long long n, long long stride,
                             int len, double dt) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const long long ia = (i / stride) % len;
    const double sg = ia < len - 1 ? 0.5 * ((double)rho0[i] + (double)rho0[i + stride]) : (double)rho0[i];
    out[i] = (float)(dt / sg);
}

// tau (and eta) of the absorption model; alpha is a map (alpha_map) or the scalar alpha_s, c0 a map
// (c0_map) or the scalar c0_s
__global__ void k_setup_absorb(const float* __restrict__ c0_map, double c0_s, const float* __restrict__ alpha_map,
                               double alpha_s, double np1, double y, int stokes, double tn, float* __restrict__ tau,
                               float* __restrict__ eta, long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double c = c0_map ? (double)c0_map[i] : c0_s;
    const double anp = (alpha_map ? (double)alpha_map[i] : alpha_s) * np1;
    if (stokes) {
        tau[i] = (float)(-2.0 * anp * c);
        return;
    }
    tau[i] = (float)(-2.0 * anp * pow(c, y - 1.0));
    if (eta) eta[i] = (float)(2.0 * anp * pow(c, y) * tn);
}

// radial tables over the half spectrum [A][B][Cp] (padding bins stay zero); kv_* are the FP64
// wavenumbers of the layout axes (a single zero for an axis of length 1)
__global__ void k_setup_radial(const double* __restrict__ kA, const double* __restrict__ kB, const double* __restrict__ kC,
                               int A, int B, int Ch, int Cp, double half, double y, float* __restrict__ kap,
                               float* __restrict__ skap, float* __restrict__ nu1, float* __restrict__ nu2) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)A * B * Ch) return;
    const int kc = (int)(q % Ch);
    const long long r = q / Ch;
    const int ib = (int)(r % B), ia = (int)(r / B);
    const size_t i = ((size_t)ia * B + ib) * Cp + kc;
    const double k = sqrt(kA[ia] * kA[ia] + kB[ib] * kB[ib] + kC[kc] * kC[kc]);
    const double arg = k * half;
    kap[i] = (float)(arg == 0.0 ? 1.0 : sin(arg) / arg);
    if (skap) skap[i] = (float)cos(arg);
    if (nu1) nu1[i] = (float)(k == 0.0 ? 0.0 : pow(k, y - 2.0));
    if (nu2) nu2[i] = (float)(k == 0.0 ? 0.0 : pow(k, y - 1.0));
}

// max of x (NaNs ignored, as std::max(m, x) with m first ignores them) as order-preserving bits:
// a float's bits with the sign bit flipped (non-negative) or all bits flipped (negative) compare
// as unsigned integers in the order of the values, so one atomicMax per warp gives the maximum
__global__ void k_setup_max(const float* __restrict__ x, long long n, unsigned int* out) {
    float m = -INFINITY;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, x[i]);
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    const unsigned b = __float_as_uint(m);
    if ((threadIdx.x & 31) == 0) atomicMax(out, (b & 0x80000000u) ? ~b : (b | 0x80000000u));
}

static unsigned blocks(long long n) { return (unsigned)((n + 255) / 256); }

void launch_setup_max(cudaStream_t st, const float* x, long long n, unsigned int* d_bits) {
    const long long b = std::min<long long>((n + 255) / 256, 148 * 8);
    k_setup_max<<<(unsigned)(b < 1 ? 1 : b), 256, 0, st>>>(x, n, d_bits);
}

float setup_max_decode(unsigned int bits) {
    const unsigned b = (bits & 0x80000000u) ? (bits & 0x7fffffffu) : ~bits;
    float f;
    std::memcpy(&f, &b, sizeof f);
    return f;
}

void launch_setup_c2(cudaStream_t st, const float* c0, float* c2, long long n) {
    k_setup_c2<<<blocks(n), 256, 0, st>>>(c0, c2, n);
}
void launch_setup_dtor(cudaStream_t st, const float* rho0, float* out, long long n, long long stride, int len, double dt) {
    k_setup_dtor<<<blocks(n), 256, 0, st>>>(rho0, out, n, stride, len, dt);
}
void launch_setup_absorb(cudaStream_t st, const float* c0_map, double c0_s, const float* alpha_map, double alpha_s,
                         double np1, double y, int stokes, double tn, float* tau, float* eta, long long n) {
    k_setup_absorb<<<blocks(n), 256, 0, st>>>(c0_map, c0_s, alpha_map, alpha_s, np1, y, stokes, tn, tau, eta, n);
}
void launch_setup_radial(cudaStream_t st, const double* kA, const double* kB, const double* kC, int A, int B, int Ch,
                         int Cp, double half, double y, float* kap, float* skap, float* nu1, float* nu2) {
    k_setup_radial<<<blocks((long long)A * B * Ch), 256, 0, st>>>(kA, kB, kC, A, B, Ch, Cp, half, y, kap, skap, nu1, nu2);
}

}  // namespace kw
