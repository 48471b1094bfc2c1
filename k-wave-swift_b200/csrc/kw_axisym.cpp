// kw_axisym.cpp — host side of the axisymmetric solver (kspaceFirstOrderAS,
// Solver/KSpaceFirstOrderAS.swift:19-309).
//
// The [nx][ny] simulation (x axial, y radial) is set up like any 2D one (medium, smoothing,
// sources, sensor; kw_engine.cpp), then given a radial PML at the outer edge only. Its spectral
// operators run on a second descriptor, the "carrier", that describes the 4x radial expansion
// [nx][4 ny]: κ and cos κ on the expanded wavenumbers, the staggered derivative and shift vectors
// of both axes, three half spectra and expanded work fields. A step mirrors the fields it needs
// into the carrier's work fields (kw_axisym.cu), runs the ordinary R2C / column / C2R passes on the
// carrier (κ ∂x⁺ and κ ∂y⁺ of p; κ ∂x⁻ of ux; κ ∂y⁻ of uy plus the κ-shifted uy / r) and takes the
// trimmed results back in the update kernels. The whole step is captured in the same CUDA graph
// as a normal step.
#include "kw_engine.h"

#include <cmath>
#include <cstring>
#include <initializer_list>
#include <utility>

namespace kw {

static std::vector<double> as_wavenumbers(int n, double d) {   // 2 pi fftfreq(n, d)
    std::vector<double> r(n);
    const double val = 1.0 / ((double)n * d);
    const int cutoff = (n - 1) / 2 + 1;
    for (int i = 0; i < cutoff; ++i) r[i] = (double)i * val;
    int j = -(n / 2);
    for (int i = cutoff; i < n; ++i) r[i] = (double)(j++) * val;
    for (auto& v : r) v *= 2.0 * M_PI;
    return r;
}

// the right (outer) ramp of the PML profile only (PML.swift:17-43 with axisymmetric: true)
static std::vector<float> as_outer_pml(int n, double dx, double dt, double c, int m, double alpha, bool staggered) {
    std::vector<float> v(n, 1.f);
    const double a = alpha * (c / dx), md = (double)m;
    for (int k = 0; k < std::min(m, n); ++k) {
        const double x = (double)(k + 1), pos = staggered ? (x + 0.5) / md : x / md;
        v[n - m + k] = (float)std::exp(-a * dt / 2.0 * std::pow(pos, 4.0));
    }
    return v;
}

void Engine::create_as_carrier() {
    SimHost& s = sims_[0];
    const kw_sim_desc& d = s.d;
    const int nx = s.B, ny = s.C, nye = 4 * ny;
    const double dx = s.d_ref[0], dy = s.d_ref[1], dt = d.dt, cref = s.cref;

    // radial PML at the outer edge only; the divergence field the density kernel keeps for the
    // Stokes term (a lossless setup has none)
    s.dev.ax[1].pml = upload(as_outer_pml(ny, dy, dt, cref, d.pml_size, d.pml_alpha, false));
    s.dev.ax[1].pml_sg = upload(as_outer_pml(ny, dy, dt, cref, d.pml_size, d.pml_alpha, true));
    if (!s.dev.div_term) s.dev.div_term = (float*)dalloc((size_t)s.N * sizeof(float));
    check(cudaMemcpyAsync(d_sims_, &s.dev, sizeof(SimDev), cudaMemcpyHostToDevice, st()), "upload sim");

    SimHost& h = car_;
    h = SimHost{};
    h.dim = 2;
    h.A = 1; h.B = nx; h.C = nye;
    h.n_ref[0] = nx; h.n_ref[1] = nye;
    h.d_ref[0] = dx; h.d_ref[1] = dy;
    h.N = (long long)nx * nye;
    h.Ch = nye / 2 + 1;
    h.Cp = (h.Ch + 3) & ~3;
    h.Ns = (long long)nx * h.Cp;
    h.M = nye / 2;
    h.nt = s.nt;
    h.cref = cref;
    h.d = d;
    h.d.record = 0;
    SimDev& v = h.dev;
    std::memset(&v, 0, sizeof(v));
    v.dim = 2; v.A = 1; v.B = nx; v.C = nye; v.Ch = h.Ch; v.Cp = h.Cp;
    v.N = h.N; v.Ns = h.Ns; v.nt = h.nt;
    v.inv_n = (float)(1.0 / (double)h.N);
    for (int L = 0; L < 3; ++L) v.axis_of_layout[L] = L - 1;
    build_plan(v.plan_row, h.M);
    build_plan(v.plan_b, nx);
    build_plan(v.plan_a, 1);
    {
        std::vector<float2> rt(nye / 2 + 1);
        for (int k = 0; k <= nye / 2; ++k) {
            const double a = -2.0 * M_PI * (double)k / (double)nye;
            rt[k] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        v.row_tw = upload(rt);
    }
    // staggered derivative and shift vectors of both axes of the expanded grid (Hermitian part at
    // the self-conjugate bin, as the main solver's)
    std::vector<std::vector<double>> kv(2);
    kv[0] = as_wavenumbers(nx, dx);
    kv[1] = as_wavenumbers(nye, dy);
    for (int a = 0; a < 2; ++a) {
        const int n = a == 0 ? nx : nye;
        const double dd = a == 0 ? dx : dy;
        std::vector<float2> dp(n), dn(n), co(n);
        for (int i = 0; i < n; ++i) {
            const double k = kv[a][i], th = k * (dd / 2.0);
            const bool nyq = (n % 2 == 0) && i == n / 2;
            dp[i] = make_float2((float)(-k * std::sin(th)), nyq ? 0.f : (float)(k * std::cos(th)));
            dn[i] = make_float2((float)(k * std::sin(th)), nyq ? 0.f : (float)(k * std::cos(th)));
            co[i] = make_float2((float)std::cos(th), nyq ? 0.f : (float)(-std::sin(th)));
        }
        AxisDev& ax = v.ax[a];
        ax.n = n;
        ax.dpos = upload(dp);
        ax.dneg = upload(dn);
        ax.colloc = upload(co);
        ax.inv_d = (float)(1.0 / dd);
    }
    // κ and cos κ on the expanded half spectrum [1][nx][Cp]
    {
        std::vector<float> kap((size_t)h.Ns, 0.f), skap((size_t)h.Ns, 0.f);
        const double half = cref * dt / 2.0;
        for (int ib = 0; ib < nx; ++ib)
            for (int kc = 0; kc < h.Ch; ++kc) {
                const double k = std::sqrt(kv[0][ib] * kv[0][ib] + kv[1][kc] * kv[1][kc]);
                const double arg = k * half;
                const size_t i = (size_t)ib * h.Cp + kc;
                kap[i] = (float)(arg == 0.0 ? 1.0 : std::sin(arg) / arg);
                skap[i] = (float)std::cos(arg);
            }
        v.radial[RT_KAPPA] = upload(kap);
        v.radial[RT_SKAPPA] = upload(skap);
    }
    const size_t fb = (size_t)h.N * sizeof(float);
    for (int k = 0; k < 3; ++k) {
        v.spec[k] = (float2*)dalloc((size_t)h.Ns * sizeof(float2));
        check(cudaMemsetAsync(v.spec[k], 0, (size_t)h.Ns * sizeof(float2), st()), "zero");
        v.tmp[k] = (float*)dalloc(fb);
    }
    v.p = (float*)dalloc(fb);
    v.rho_sum = (float*)dalloc(fb);
    for (int a = 0; a < 2; ++a) {
        v.u[a] = (float*)dalloc(fb);
        v.rho[a] = (float*)dalloc(fb);
    }
    v.nonfinite = d_flag_;
    v.wait_cycles = wait_cycles_;
    v.test_stall = test_stall_;
    build_tensor_maps(h, v);
    d_car_ = (SimDev*)dalloc(sizeof(SimDev));
    check(cudaMemcpyAsync(d_car_, &v, sizeof(SimDev), cudaMemcpyHostToDevice, st()), "upload sim");
    // the setup's smoothing jobs cached tile maps of the [nx][ny] geometry; the spectral jobs from
    // here on are the carrier's
    maps_.clear();
    as_mode_ = true;
}

void Engine::issue_step_as(bool first) {
    SimHost& s = sims_[0];
    const SimDev& sv = s.dev;
    const SimDev& cv = car_.dev;
    const long long n = s.N, ne = car_.N;
    const int nye = car_.C;
    // spectral jobs run on the carrier: the pass launchers read sims_ and d_sims_
    auto job = [&](int in_field, int nin, int fanout, int nout, std::initializer_list<OpSpec> ops, int out_field,
                   const char* name) {
        SpecJob j;
        j.in_field = in_field;
        j.nin = nin;
        j.fanout = fanout;
        j.nout = nout;
        int c = 0;
        for (const OpSpec& o : ops) j.op[c++] = o;
        j.spec_in = 0;
        j.spec_out = 0;
        j.epi = EPI_STORE;
        j.out_field = out_field;
        j.name = name;
        std::swap(sims_[0], car_);
        std::swap(d_sims_, d_car_);
        auto back = [&] {
            std::swap(sims_[0], car_);
            std::swap(d_sims_, d_car_);
        };
        try {
            issue_job(j, -1);
        } catch (...) {
            back();
            throw;
        }
        back();
    };
    auto mirror = [&](const float* src, float* dst, int kind, int over_r) {
        launch_as_mirror(st(), d_sims_, d_car_, ne, src, dst, kind, over_r);
    };
    const OpSpec xpos{AO_DPOS, 0, RT_KAPPA, 0}, ypos{AO_DPOS, 1, RT_KAPPA, 0};
    auto gradients_to_velocity = [&](int init) {   // κ ∂⁺ of the WSWA-mirrored p
        mirror(sv.p, cv.p, AS_WSWA, 0);
        job(FS_P, 1, 1, 2, {xpos, ypos}, FS_TMP, "as_grad");
        launch_as_vel(st(), d_sims_, n, cv.tmp[0], cv.tmp[1], nye, init);
    };
    // additive sources: the scaled values in a sparse field, mirrored and filtered by cos κ
    auto corrected = [&](float* buf, int kind, float* f0, float* f1) {
        mirror(buf, cv.p, kind, 0);
        job(FS_P, 1, 0, 1, {OpSpec{AO_NONE, 0, RT_SKAPPA, 0}}, FS_TMP, "as_src");
        launch_as_add(st(), d_sims_, n, cv.tmp[0], nye, f0, f1);
    };

    // velocity (KSpaceFirstOrderAS.swift:254-259)
    gradients_to_velocity(0);
    for (int a = 0; a < 2; ++a) {
        const SourceDev& us = sv.usrc[a];
        if (us.nsrc <= 0 || us.len <= 0) continue;
        launch_as_src(st(), d_sims_, d_t_, us.nsrc, 1 + a, us.mode == KW_SOURCE_ADDITIVE ? sv.src_buf[a] : nullptr);
        if (us.mode == KW_SOURCE_ADDITIVE) corrected(sv.src_buf[a], a == 0 ? AS_WSWA : AS_HAHS, sv.u[a], nullptr);
    }
    // divergence: κ ∂x⁻ WSWA(ux); κ e^{-ik dy/2} (i ky HAHS(uy) + HSHA(uy / r)) (:262-267)
    mirror(sv.u[0], cv.p, AS_WSWA, 0);
    mirror(sv.u[1], cv.u[0], AS_HAHS, 0);
    mirror(sv.u[1], cv.u[1], AS_HSHA, 1);
    job(FS_P, 1, 0, 1, {OpSpec{AO_DNEG, 0, RT_KAPPA, 0}}, FS_TMP, "as_divx");
    job(FS_U, 2, 0, 2, {OpSpec{AO_DNEG, 1, RT_KAPPA, 0}, OpSpec{AO_COLLOC, 1, RT_KAPPA, 1}}, FS_RHO, "as_divy");
    launch_as_den(st(), d_sims_, n, cv.tmp[0], cv.rho[0], cv.rho[1], nye);
    // pressure source into both density splits (:281-300)
    const SourceDev& ps = sv.psrc;
    if (ps.nsrc > 0 && ps.len > 0) {
        launch_as_src(st(), d_sims_, d_t_, ps.nsrc, 0, ps.mode == KW_SOURCE_ADDITIVE ? sv.src_buf[0] : nullptr);
        if (ps.mode == KW_SOURCE_ADDITIVE) corrected(sv.src_buf[0], AS_WSWA, sv.rho[0], sv.rho[1]);
    }
    launch_as_eos(st(), d_sims_, n);
    // t = 0 override for an initial pressure (:311-318)
    if (first && s.p0s) {
        launch_as_p0(st(), d_sims_, n, s.p0s);
        gradients_to_velocity(1);
    }
    if (any_recp_) timed("sample_p", 0, [&] { launch_sample(st(), d_sims_, d_t_, count(), max_pts_, 0, 0); });
    timed("tick", 0, [&] { launch_tick(st(), d_t_); });
}

}  // namespace kw
