// kw_derivative.cpp — the staggered spectral derivative of one device field, run through the
// same pass kernels as the time step:
//   out = Re F^-1( i k_a exp(s i k_a d_a / 2) F(in) ),  s = +1 or -1,
// i.e. the reference's derivativeOperator (Sources/KWave/Solver/KSpaceFirstOrder.swift:764-769)
// applied on its own (the time step multiplies it by kappa as well). The half-spectrum lives in a
// scratch buffer obtained through the engine's allocator.
#include "kw_engine.h"

#include <cmath>
#include <cstring>

namespace kw {

static std::vector<double> wavenumber_vec(int n, double d) {   // 2 pi fftfreq(n, d)
    std::vector<double> r(n);
    const double val = 1.0 / ((double)n * d);
    const int cutoff = (n - 1) / 2 + 1;
    for (int i = 0; i < cutoff; ++i) r[i] = (double)i * val;
    int j = -(n / 2);
    for (int i = cutoff; i < n; ++i) r[i] = (double)(j++) * val;
    for (auto& v : r) v *= 2.0 * M_PI;
    return r;
}

void Engine::create_derivative(int dim, const int* n, const double* d, int axis, int shift, const float* in,
                               float* out) {
    if (dim < 1 || dim > 3) throw KwError{KW_ERR_INVALID, "dim must be 1, 2 or 3"};
    if (axis < 0 || axis >= dim) throw KwError{KW_ERR_INVALID, "axis must be in [0, dim)"};
    if (shift != 1 && shift != -1) throw KwError{KW_ERR_INVALID, "shift must be +1 or -1"};
    if (!in || !out) throw KwError{KW_ERR_INVALID, "null field pointer"};
    for (int a = 0; a < dim; ++a) {
        if (n[a] < 1 || n[a] > 4096) throw KwError{KW_ERR_UNSUPPORTED, "axis lengths must be in [1, 4096]"};
        if (!(d[a] > 0)) throw KwError{KW_ERR_INVALID, "grid spacing must be positive"};
    }
    check(cudaSetDevice(ctx_->device), "cudaSetDevice");
    sims_.resize(1);
    outs_.resize(1);
    dim_ = dim;
    SimHost& h = sims_[0];
    h.dim = dim;
    for (int a = 0; a < dim; ++a) { h.n_ref[a] = n[a]; h.d_ref[a] = d[a]; }
    if (dim == 1) { h.A = 1; h.B = 1; h.C = n[0]; }
    else if (dim == 2) { h.A = 1; h.B = n[0]; h.C = n[1]; }
    else { h.A = n[0]; h.B = n[1]; h.C = n[2]; }
    h.N = (long long)h.A * h.B * h.C;
    h.Ch = h.C / 2 + 1;
    h.Cp = (h.Ch + 3) & ~3;   // a multiple of 4 (16-byte rows of the float radial tables)
    h.Ns = (long long)h.A * h.B * h.Cp;
    h.M = (h.C & 1) ? h.C : h.C / 2;
    h.nt = 1;
    h.d.record = 0;

    d_sims_ = (SimDev*)dalloc(sizeof(SimDev));
    d_t_ = (int*)dalloc(sizeof(int));
    d_flag_ = (int*)dalloc(2 * sizeof(int));
    d_red_ = (unsigned int*)dalloc(4 * sizeof(unsigned int));
    d_p0s_ = (const float**)dalloc(sizeof(float*));

    SimDev& v = h.dev;
    std::memset(&v, 0, sizeof(v));
    v.dim = dim; v.A = h.A; v.B = h.B; v.C = h.C; v.Ch = h.Ch; v.Cp = h.Cp;
    v.N = h.N; v.Ns = h.Ns; v.nt = 1;
    v.inv_n = (float)(1.0 / (double)h.N);
    for (int L = 0; L < 3; ++L) v.axis_of_layout[L] = L + dim - 3;
    build_plan(v.plan_row, h.M);
    build_plan(v.plan_b, h.B);
    build_plan(v.plan_a, h.A);
    {
        std::vector<float2> rt(h.C / 2 + 1);
        for (int k = 0; k <= h.C / 2; ++k) {
            const double a = -2.0 * M_PI * (double)k / (double)h.C;
            rt[k] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        v.row_tw = upload(rt);
    }
    for (int a = 0; a < dim; ++a) v.ax[a].n = n[a];
    {
        // i k exp(s i k d / 2), Hermitian (real part) at the Nyquist bin of an even axis
        const int na = n[axis];
        const double da = d[axis];
        const std::vector<double> kv = wavenumber_vec(na, da);
        std::vector<float2> op(na);
        for (int i = 0; i < na; ++i) {
            const double k = kv[i], th = k * (da / 2.0);
            const bool nyq = (na % 2 == 0) && i == na / 2;
            op[i] = make_float2((float)(-shift * k * std::sin(th)), nyq ? 0.f : (float)(k * std::cos(th)));
        }
        float2* dv = upload(op);
        if (shift > 0) v.ax[axis].dpos = dv;
        else v.ax[axis].dneg = dv;
    }
    v.spec[0] = (float2*)dalloc((size_t)h.Ns * sizeof(float2));
    v.p = const_cast<float*>(in);
    v.tmp[0] = out;
    v.nonfinite = d_flag_;
    v.wait_cycles = wait_cycles_;
    v.test_stall = test_stall_;
    build_tensor_maps(h, v);
    check(cudaMemcpyAsync(d_sims_, &v, sizeof(SimDev), cudaMemcpyHostToDevice, st()), "upload sim");
    deriv_axis_ = axis;
    deriv_shift_ = shift;
    t_ = 0;
}

void Engine::run_derivative() {
    SpecJob j;
    j.in_field = FS_P;
    j.nin = 1;
    j.nout = 1;
    j.op[0] = OpSpec{(int8_t)(deriv_shift_ > 0 ? AO_DPOS : AO_DNEG), (int8_t)deriv_axis_, RT_NONE, 0};
    j.spec_in = 0;
    j.spec_out = 0;
    j.epi = EPI_STORE;
    j.out_field = FS_TMP;
    j.name = "deriv";
    issue_job(j, -1);
    check(cudaGetLastError(), "launch");
    check(cudaStreamSynchronize(st()), "derivative sync");
    check_kernel_error();
}

}  // namespace kw
