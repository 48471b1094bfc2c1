/*
 * kwref.cpp — FP64 CPU ORACLE for the k-space pseudospectral fluid time loop.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA library: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it. The product library never
 * links, loads or calls it.
 *
 * It restates, in double precision and in plain loops, the algorithm of k-wave-swift
 * (paths are relative to that project):
 *   Sources/KWave/Solver/KSpaceFirstOrder.swift   (KSFO) 79-907   solver, operators, absorption
 *   Sources/KWave/Sensor/Recording.swift          (REC)  1-168    sensor sampling, aggregates
 *   Sources/KWave/PML/PML.swift                   (PML)  17-43    pmlProfile
 *   Sources/KWave/Filter/Filters.swift            (FILT) 202-347  smooth / smooth1D / smooth3D
 *   Sources/KWave/Grid/KWaveGrid.swift            (GRID) 67-101   wavenumbers
 *   Sources/KWave/Internal/Support.swift                   6-19   fftFreq
 *   Sources/KWave/Material/Conversion.swift                6-8    db2neper
 *   Sources/KWave/Sensor/Directivity.swift                 14-79  2D sensor directivity
 * Every transform is a full complex DFT followed by the real part, exactly like the
 * reference's MLXFFT.fftn(...).realPart() chains; nothing is reordered or fused.
 *
 * Parity status: UNPINNED against reference outputs. k-wave-swift ships no golden data (its
 * parity fixtures are generated by k-wave-python, which is absent), and the Swift/MLX package
 * cannot be built here. The oracle is pinned instead to the reference's own known-answer and
 * self-consistency tests (Tests/KWaveTests/SolverTests.swift, FFTTests.swift, GridTests.swift,
 * UtilTests.swift, ParityTests.swift:63) and cross-checked against an independent numpy
 * restatement (tests/golden/make_golden.py).
 */
#include "../include/kwave_cuda.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using cd = std::complex<double>;
using vecd = std::vector<double>;
using vecc = std::vector<cd>;

static thread_local std::string g_err;

/* ======================================================================================
 * FFT: recursive mixed-radix decimation in time, any length (prime factors handled by a
 * direct DFT of that factor). Forward = exp(-2 pi i jk/n), inverse unnormalised.
 * ====================================================================================== */
struct FFTPlan {
    int n = 0;
    std::vector<int> fac;
    vecc tw;  // tw[j] = exp(-2 pi i j / n)
    explicit FFTPlan(int n_) : n(n_) {
        int m = n;
        for (int p : {4, 2, 3, 5}) {
            while (m % p == 0) { fac.push_back(p); m /= p; }
        }
        for (int p = 7; m > 1; p += 2) {
            while (m % p == 0) { fac.push_back(p); m /= p; }
            if (p * p > m && m > 1) { fac.push_back(m); m = 1; }
        }
        tw.resize(n);
        for (int j = 0; j < n; ++j) {
            double a = -2.0 * M_PI * (double)j / (double)n;
            tw[j] = cd(std::cos(a), std::sin(a));
        }
    }
};

static void fft_rec(const FFTPlan& pl, const cd* in, ptrdiff_t istride, cd* out, int n,
                    const int* fac, bool inv, cd* scratch) {
    if (n == 1) { out[0] = in[0]; return; }
    const int p = fac[0];
    const int m = n / p;
    for (int q = 0; q < p; ++q)
        fft_rec(pl, in + q * istride, istride * p, out + (size_t)q * m, m, fac + 1, inv, scratch);
    const int step = pl.n / n;  // W_n^j = tw[j * step]
    for (int k = 0; k < m; ++k) {
        for (int q = 0; q < p; ++q) {
            cd w = pl.tw[((size_t)q * k * step) % pl.n];
            if (inv) w = std::conj(w);
            scratch[q] = out[(size_t)q * m + k] * w;
        }
        for (int s = 0; s < p; ++s) {
            cd acc = 0.0;
            for (int q = 0; q < p; ++q) {
                cd w = pl.tw[((size_t)q * s * m * step) % pl.n];  // W_p^{qs}
                if (inv) w = std::conj(w);
                acc += scratch[q] * w;
            }
            out[(size_t)s * m + k] = acc;
        }
    }
}

static void fft1d(const FFTPlan& pl, cd* data, bool inv) {
    static thread_local std::vector<cd> tmp, scratch;
    tmp.assign(data, data + pl.n);
    scratch.resize(pl.fac.empty() ? 1 : (size_t)*std::max_element(pl.fac.begin(), pl.fac.end()));
    fft_rec(pl, tmp.data(), 1, data, pl.n, pl.fac.data(), inv, scratch.data());
}

struct Shape {
    int dim = 1;
    int n[3] = {1, 1, 1};
    double d[3] = {1, 1, 1};
    size_t N = 1;
    size_t stride[3] = {1, 1, 1};
    void finish() {
        N = 1;
        for (int a = dim - 1; a >= 0; --a) { stride[a] = N; N *= (size_t)n[a]; }
    }
    int idx(size_t flat, int a) const { return (int)((flat / stride[a]) % (size_t)n[a]); }
};

/* n-D complex FFT in place (MLXFFT.fft / fft2 / fftn), unnormalised forward,
 * inverse scaled by 1/N like ifftn. */
static void fftn(const Shape& s, vecc& x, bool inv) {
    for (int a = 0; a < s.dim; ++a) {
        const int n = s.n[a];
        const size_t st = s.stride[a];
        const size_t nlines = s.N / n;
        FFTPlan pl(n);
#pragma omp parallel
        {
            std::vector<cd> line(n);
#pragma omp for schedule(static)
            for (long long L = 0; L < (long long)nlines; ++L) {
                // line L: base = (L / st) * st * n + (L % st)
                size_t base = ((size_t)L / st) * st * n + ((size_t)L % st);
                for (int i = 0; i < n; ++i) line[i] = x[base + (size_t)i * st];
                fft1d(pl, line.data(), inv);
                for (int i = 0; i < n; ++i) x[base + (size_t)i * st] = line[i];
            }
        }
    }
    if (inv) {
        const double sc = 1.0 / (double)s.N;
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)s.N; ++i) x[i] *= sc;
    }
}

static vecc to_complex(const vecd& f) {
    vecc c(f.size());
    for (size_t i = 0; i < f.size(); ++i) c[i] = cd(f[i], 0.0);
    return c;
}

/* ======================================================================================
 * Host setup helpers (restated in FP64)
 * ====================================================================================== */

// Support.swift:6-19 — 2*pi*fftfreq(n, d)
static vecd wavenumber_vector(int n, double d) {
    vecd r(n);
    const double val = 1.0 / ((double)n * d);
    const int cutoff = (n - 1) / 2 + 1;
    for (int i = 0; i < cutoff; ++i) r[i] = (double)i * val;
    int j = -(n / 2);
    for (int i = cutoff; i < n; ++i) { r[i] = (double)j * val; ++j; }
    for (auto& v : r) v *= 2.0 * M_PI;
    return r;
}

// PML.swift:17-43
static vecd pml_profile(int n, double dx, double dt, double c, int m, double alpha, bool staggered) {
    const double power = 4.0;
    const double a = alpha * (c / dx);
    const double md = (double)m;
    vecd pml(n, 1.0);
    for (int k = 0; k < std::min(m, n); ++k) {
        const double x = (double)(k + 1);
        double posL, posR;
        if (staggered) { posL = (md + 0.5 - x) / md; posR = (x + 0.5) / md; }
        else { posL = (md + 1.0 - x) / md; posR = x / md; }
        pml[k] = std::exp(-a * dt / 2.0 * std::pow(posL, power));
        pml[n - m + k] = std::exp(-a * dt / 2.0 * std::pow(posR, power));
    }
    return pml;
}

// Filters.swift:203-210 symmetric Blackman window
static vecd blackman1d(int n) {
    if (n <= 1) return vecd(std::max(n, 0), 1.0);
    vecd w(n);
    const double denom = (double)(n - 1);
    for (int i = 0; i < n; ++i) {
        const double x = 2.0 * M_PI * (double)i / denom;
        w[i] = 0.42 - 0.5 * std::cos(x) + 0.08 * std::cos(2.0 * x);
    }
    return w;
}

// Filters.swift:264-269 (and the identical inline interp of rotationWindow2D, 232-238)
static double interp_radial(double r, const vecd& win, double radius) {
    const double pos = std::min(r, radius) + radius;
    const int i0 = std::min((int)std::floor(pos), (int)win.size() - 2);
    const double frac = pos - (double)i0;
    return std::fabs(win[i0] * (1.0 - frac) + win[i0 + 1] * frac);
}

/* The k-space smoothing window in FFT order for a field of this shape, element by element the
 * array the reference multiplies the spectrum with:
 *   1D smooth1D  FILT:273-292, 2D smooth FILT:218-249 + 325-338, 3D smooth3D FILT:295-315.
 * The 2D variant fills out[i][j] = win[(i+sx)%nx][(j+sy)%ny]; the 1D/3D variants fill
 * out[(i+sx)%n] = win[i]; both are kept literally (they differ only for odd sizes). */
static vecd smoothing_window(const Shape& s) {
    std::vector<int> sizes(s.n, s.n + s.dim), enlarged(s.dim);
    int L = 1;
    for (int a = 0; a < s.dim; ++a) { enlarged[a] = sizes[a] % 2 != 0 ? sizes[a] : sizes[a] + 1; L = std::max(L, enlarged[a]); }
    const vecd winLin = blackman1d(L);
    const double radius = (double)(L - 1) / 2.0;
    std::vector<vecd> axes(s.dim);
    for (int a = 0; a < s.dim; ++a) {
        const int cnt = enlarged[a];
        if (cnt <= 1) { axes[a] = vecd(1, 0.0); continue; }
        axes[a].resize(cnt);
        for (int i = 0; i < cnt; ++i) axes[a][i] = -radius + 2.0 * radius * (double)i / (double)(cnt - 1);
    }
    vecd out(s.N, 0.0);
    if (s.dim == 2) {
        const int nx = s.n[0], ny = s.n[1];
        const int sx = (nx + 1) / 2, sy = (ny + 1) / 2;
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                const int wi = (i + sx) % nx, wj = (j + sy) % ny;
                const double r = std::sqrt(axes[0][wi] * axes[0][wi] + axes[1][wj] * axes[1][wj]);
                out[(size_t)i * ny + j] = interp_radial(r, winLin, radius);
            }
    } else if (s.dim == 3) {
        const int nx = s.n[0], ny = s.n[1], nz = s.n[2];
        const int sx = (nx + 1) / 2, sy = (ny + 1) / 2, sz = (nz + 1) / 2;
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k) {
                    const double r = std::sqrt(axes[0][i] * axes[0][i] + axes[1][j] * axes[1][j] + axes[2][k] * axes[2][k]);
                    const int di = (i + sx) % nx, dj = (j + sy) % ny, dk = (k + sz) % nz;
                    out[((size_t)di * ny + dj) * nz + dk] = interp_radial(r, winLin, radius);
                }
    } else {
        const int nx = s.n[0];
        const int sx = (nx + 1) / 2;
        for (int i = 0; i < nx; ++i) out[(i + sx) % nx] = interp_radial(std::fabs(axes[0][i]), winLin, radius);
    }
    return out;
}

// smooth(a, restore_max) — Re(ifftn(W * fftn(f))) * max|f| / max|out|
static vecd smooth_field(const Shape& s, const vecd& f) {
    const vecd w = smoothing_window(s);
    vecc F = to_complex(f);
    fftn(s, F, false);
    for (size_t i = 0; i < s.N; ++i) F[i] *= w[i];
    fftn(s, F, true);
    vecd out(s.N);
    double srcMax = 0, outMax = 0;
    for (size_t i = 0; i < s.N; ++i) {
        out[i] = F[i].real();
        srcMax = std::max(srcMax, std::fabs(f[i]));
        outMax = std::max(outMax, std::fabs(out[i]));
    }
    const double scale = outMax > 0 ? srcMax / outMax : 1.0;
    for (auto& v : out) v *= scale;
    return out;
}

// Conversion.swift:6-8
static double db2neper(double alpha, double y) {
    return 100.0 * alpha * std::pow(1e-6 / (2.0 * M_PI), y) / (20.0 * std::log10(M_E));
}

/* ======================================================================================
 * The simulation
 * ====================================================================================== */
struct SourceOp {                      // KSFO:129-175
    std::vector<size_t> idx;
    std::vector<std::vector<double>> signal;  // [rows][len]
    vecd scale;
    int mode = KW_SOURCE_ADDITIVE;
    int len() const { return signal.empty() ? 0 : (int)signal[0].size(); }
};

struct kwref_result {
    Shape s;
    int nt = 0, steps = 0;
    int nsensor = 0;
    unsigned record = 0;
    bool have_p_series = false, have_u_series = false;
    std::vector<vecd> fields;          // indexed by kw_field
    std::vector<int> present;          // element count > 0 when present
    double loop_seconds = 0;
};

static bool fail(const std::string& m) { g_err = m; return false; }

static bool grid_sized(const kw_array& a, size_t N) { return a.data && (a.len == 1 || a.len == N); }

static vecd expand(const kw_array& a, size_t N) {
    vecd v(N);
    for (size_t i = 0; i < N; ++i) v[i] = (double)(a.len == 1 ? a.data[0] : a.data[i]);
    return v;
}

// KSFO:778-782 flatNonzeroIndices
static std::vector<size_t> flat_nonzero(const float* mask, size_t N) {
    std::vector<size_t> r;
    for (size_t i = 0; i < N; ++i) if (mask[i] != 0.0f) r.push_back(i);
    return r;
}

// KSFO:799-806 staggerDensity along axis a (edge replicated)
static vecd stagger_density(const Shape& s, const vecd& rho, int a) {
    vecd out(s.N);
    const size_t st = s.stride[a];
    const int n = s.n[a];
    for (size_t i = 0; i < s.N; ++i) {
        const int ia = s.idx(i, a);
        out[i] = ia < n - 1 ? 0.5 * (rho[i] + rho[i + st]) : rho[i];
    }
    return out;
}

/* ======================================================================================
 * The model: everything kspaceFirstOrder precomputes before its time loop (KSFO:203-442),
 * shared by the forward run and the discrete adjoint.
 * ====================================================================================== */
struct DirEntry { vecd weight; std::vector<int> rows; std::vector<size_t> gather; };

struct Model {
    Shape s;
    size_t N = 0;
    int ndim = 1;
    double dt = 0;
    int nt = 0;
    vecd c0, rho0, c2, dtRho0;
    double cRef = 0;
    std::vector<vecd> kv;
    vecd kmag, kappa, skappa;
    std::vector<vecc> ddPos, ddNeg, colloc;
    std::vector<vecd> pml, pmlSg, dtOverRho;
    std::vector<SourceOp> pOp, uOp;
    std::vector<bool> hasP, hasU;
    bool hasP0 = false;
    vecd p0f;
    bool absorb = false, stokes = false, dispersion = false;
    double y = 1.5;
    vecd tau, eta, nabla1, nabla2;
    bool nonlinear = false;
    vecd bona;
    unsigned rec = 0;
    bool recordP = false, recordU = false, recordUFinal = false;
    bool haveSampler = false;
    int nPts = 0, nCorners = 1;
    std::vector<size_t> sIdx;
    vecd sW;
    bool directivity = false;
    std::vector<DirEntry> dirEntries;
};

// The fields the time loop carries (KSFO:438-442) plus the step's intermediates.
struct State {
    vecd p, rhoTot, divU;
    std::vector<vecd> u, rho, dU;
    void init(const Model& m) {
        p.assign(m.N, 0.0);
        rhoTot.assign(m.N, 0.0);
        divU.assign(m.N, 0.0);
        u.assign(m.ndim, vecd(m.N, 0.0));
        rho.assign(m.ndim, vecd(m.N, 0.0));
        dU.assign(m.ndim, vecd(m.N, 0.0));
    }
};

// Re F^-1(H F x) for a full-grid multiplier H(i) (the reference's fftn(...).realPart() chain)
template <class HF>
static void apply_op(const Model& m, const vecd& x, vecd& out, HF H) {
    vecc w = to_complex(x);
    fftn(m.s, w, false);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < (long long)m.N; ++i) w[i] *= H((size_t)i);
    fftn(m.s, w, true);
    out.resize(m.N);
    for (size_t i = 0; i < m.N; ++i) out[i] = w[i].real();
}

static int build_model(const kw_sim_desc* d, Model& m) {
    Shape& s = m.s;
    s.dim = d->dim;
    if (s.dim < 1 || s.dim > 3) { g_err = "dim must be 1, 2 or 3"; return KW_ERR_INVALID; }
    const int ns[3] = {d->nx, d->ny, d->nz};
    const double ds[3] = {d->dx, d->dy, d->dz};
    for (int a = 0; a < s.dim; ++a) { s.n[a] = ns[a]; s.d[a] = ds[a]; if (ns[a] < 1) { g_err = "bad size"; return KW_ERR_INVALID; } }
    s.finish();
    const size_t N = s.N;
    m.N = N;
    const int ndim = s.dim;
    m.ndim = ndim;
    const double dt = d->dt;
    m.dt = dt;
    m.nt = d->nt;
    if (m.nt <= 0) { g_err = "call grid.makeTime(...) before running the solver"; return KW_ERR_INVALID; }
    if (!d->p0 && !d->p_mask && !d->u_mask) { g_err = "solver requires source.p0 or a time-varying p/u source"; return KW_ERR_INVALID; }
    if (!grid_sized(d->sound_speed, N) || !grid_sized(d->density, N)) { g_err = "soundSpeed/density must be scalar or grid-shaped"; return KW_ERR_INVALID; }
    if (d->pml_size < 0) { g_err = "bad pml size"; return KW_ERR_INVALID; }
    for (int a = 0; a < ndim; ++a) if (d->pml_size > s.n[a]) { g_err = "pml larger than grid"; return KW_ERR_INVALID; }

    // ---- medium (KSFO:367-373) ----
    const bool c0Map = d->sound_speed.len > 1, rho0Map = d->density.len > 1;
    m.c0 = expand(d->sound_speed, N);
    m.rho0 = expand(d->density, N);
    if (d->smooth_c0 && c0Map) m.c0 = smooth_field(s, m.c0);
    if (d->smooth_rho0 && rho0Map) m.rho0 = smooth_field(s, m.rho0);
    const vecd& c0 = m.c0;
    const vecd& rho0 = m.rho0;
    double cRef = 0;
    for (size_t i = 0; i < N; ++i) cRef = std::max(cRef, c0[i]);   // referenceSoundSpeed KSFO:786-788
    if (!c0Map) cRef = c0[0];
    if (!std::isnan(d->c_ref)) cRef = d->c_ref;
    m.cRef = cRef;

    // ---- k-space operators (KSFO:376-383, 764-769) ----
    m.kv.resize(ndim);
    for (int a = 0; a < ndim; ++a) m.kv[a] = wavenumber_vector(s.n[a], s.d[a]);
    m.kmag.resize(N); m.kappa.resize(N); m.skappa.resize(N);
    for (size_t i = 0; i < N; ++i) {
        double k2 = 0;
        for (int a = 0; a < ndim; ++a) { const double k = m.kv[a][s.idx(i, a)]; k2 += k * k; }
        m.kmag[i] = std::sqrt(k2);
        const double arg = m.kmag[i] * (cRef * dt / 2.0);
        m.kappa[i] = arg == 0.0 ? 1.0 : std::sin(arg) / arg;
        m.skappa[i] = std::cos(arg);
    }
    m.ddPos.resize(ndim); m.ddNeg.resize(ndim); m.colloc.resize(ndim);
    const cd I(0, 1);
    for (int a = 0; a < ndim; ++a) {
        const int n = s.n[a];
        m.ddPos[a].resize(n); m.ddNeg[a].resize(n); m.colloc[a].resize(n);
        for (int i = 0; i < n; ++i) {
            const double k = m.kv[a][i], th = k * (s.d[a] / 2.0);
            m.ddPos[a][i] = I * k * (std::cos(th) + 1.0 * I * std::sin(th));
            m.ddNeg[a][i] = I * k * (std::cos(th) - 1.0 * I * std::sin(th));
            m.colloc[a][i] = std::cos(th) - I * std::sin(th);   // REC:101-104
        }
    }

    // ---- PML (KSFO:385-397) ----
    m.pml.resize(ndim); m.pmlSg.resize(ndim);
    for (int a = 0; a < ndim; ++a) {
        m.pml[a] = pml_profile(s.n[a], s.d[a], dt, cRef, d->pml_size, d->pml_alpha, false);
        m.pmlSg[a] = pml_profile(s.n[a], s.d[a], dt, cRef, d->pml_size, d->pml_alpha, true);
    }

    // ---- staggered density etc. (KSFO:399-402) ----
    m.c2.resize(N); m.dtRho0.resize(N);
    for (size_t i = 0; i < N; ++i) { m.c2[i] = c0[i] * c0[i]; m.dtRho0[i] = dt * rho0[i]; }
    m.dtOverRho.resize(ndim);
    for (int a = 0; a < ndim; ++a) {
        vecd sg = rho0Map ? stagger_density(s, rho0, a) : rho0;
        m.dtOverRho[a].resize(N);
        for (size_t i = 0; i < N; ++i) m.dtOverRho[a][i] = dt / sg[i];
    }

    // ---- sources (KSFO:404-423, 129-201) ----
    const double nd = (double)ndim;
    // makeSourceOp KSFO:192-201: no op when the mask or the signal is absent or the mask is empty.
    auto make_op = [&](const float* mask, const kw_signal& sig, int mode, bool isP, int a, SourceOp& op) -> int {
        if (!mask || !sig.data) return 0;
        op.idx = flat_nonzero(mask, N);
        if (op.idx.empty()) return 0;
        const int rows = sig.rows, len = sig.len;
        if ((rows != 1 && rows != (int)op.idx.size()) || len < 0) return -1;
        op.signal.assign(rows, vecd(len));
        for (int r = 0; r < rows; ++r)
            for (int t = 0; t < len; ++t) op.signal[r][t] = sig.data[(size_t)r * len + t];
        op.mode = mode;
        op.scale.resize(op.idx.size());
        for (size_t q = 0; q < op.idx.size(); ++q) {
            const double c = c0[op.idx[q]];   // soundSpeedSamples KSFO:791-794
            if (isP) op.scale[q] = mode == KW_SOURCE_DIRICHLET ? 1.0 / (nd * c * c) : 2.0 * dt / (nd * c * s.d[a]);
            else op.scale[q] = mode == KW_SOURCE_DIRICHLET ? 1.0 : 2.0 * c * dt / s.d[a];
        }
        return 1;
    };
    m.pOp.assign(ndim, SourceOp()); m.uOp.assign(ndim, SourceOp());
    m.hasP.assign(ndim, false); m.hasU.assign(ndim, false);
    const kw_signal* usig[3] = {&d->ux, &d->uy, &d->uz};
    for (int a = 0; a < ndim; ++a) {
        const int rp = make_op(d->p_mask, d->p, d->p_mode, true, a, m.pOp[a]);
        const int ru = make_op(d->u_mask, *usig[a], d->u_mode, false, a, m.uOp[a]);
        if (rp < 0 || ru < 0) { g_err = "source signal rows must be 1 or the number of source points"; return KW_ERR_INVALID; }
        m.hasP[a] = rp > 0; m.hasU[a] = ru > 0;
    }

    // ---- p0 (KSFO:425-430) ----
    m.hasP0 = d->p0 != nullptr;
    if (m.hasP0) {
        m.p0f.assign(d->p0, d->p0 + N);
        if (d->smooth_p0) m.p0f = smooth_field(s, m.p0f);
    }

    // ---- absorption (KSFO:812-882) and nonlinearity (KSFO:889-907) ----
    if (d->alpha_coeff.data && d->alpha_mode != KW_ABSORPTION_NONE) {
        if (!grid_sized(d->alpha_coeff, N)) { g_err = "alphaCoeff must be scalar or grid-shaped"; return KW_ERR_INVALID; }
        m.absorb = true;
        double y = std::isnan(d->alpha_power) ? 1.5 : d->alpha_power;
        if (d->alpha_mode == KW_ABSORPTION_STOKES) y = 2.0;
        m.y = y;
        const double np1 = db2neper(1.0, y);
        vecd alphaNp = expand(d->alpha_coeff, N);
        for (auto& v : alphaNp) v *= np1;
        m.stokes = d->alpha_mode == KW_ABSORPTION_STOKES || std::fabs(y - 2.0) < 1e-10;
        m.tau.resize(N);
        if (m.stokes) {
            for (size_t i = 0; i < N; ++i) m.tau[i] = -2.0 * alphaNp[i] * c0[i];
        } else {
            m.nabla1.resize(N);
            for (size_t i = 0; i < N; ++i) {
                m.tau[i] = -2.0 * alphaNp[i] * std::pow(c0[i], y - 1.0);
                m.nabla1[i] = m.kmag[i] == 0.0 ? 0.0 : std::pow(m.kmag[i], y - 2.0);
            }
        }
        if (!m.stokes && d->alpha_mode != KW_ABSORPTION_NO_DISPERSION) {
            m.dispersion = true;
            m.eta.resize(N); m.nabla2.resize(N);
            const double tn = std::tan(M_PI * y / 2.0);
            for (size_t i = 0; i < N; ++i) {
                m.eta[i] = 2.0 * alphaNp[i] * std::pow(c0[i], y) * tn;
                m.nabla2[i] = m.kmag[i] == 0.0 ? 0.0 : std::pow(m.kmag[i], y - 1.0);
            }
        }
    }
    if (d->b_on_a.data) {
        if (!grid_sized(d->b_on_a, N)) { g_err = "bOnA must be scalar or grid-shaped"; return KW_ERR_INVALID; }
        m.bona = expand(d->b_on_a, N);
        double mx = 0;
        for (double v : m.bona) mx = std::max(mx, std::fabs(v));
        m.nonlinear = mx != 0.0;
    }

    // ---- sensor (REC:8-97) ----
    const unsigned rec = d->record;
    m.rec = rec;
    m.recordP = (rec & (KW_RECORD_P | KW_RECORD_P_MAX | KW_RECORD_P_MIN | KW_RECORD_P_RMS | KW_RECORD_I_AVG)) != 0;
    m.recordU = (rec & (KW_RECORD_UX | KW_RECORD_UY | KW_RECORD_UZ | KW_RECORD_U_MAX | KW_RECORD_U_RMS | KW_RECORD_I_AVG)) != 0;
    m.recordUFinal = (rec & KW_RECORD_U_FINAL) != 0;
    if (d->sensor_kind == KW_SENSOR_BINARY && d->sensor_mask) {
        m.haveSampler = true;
        m.sIdx = flat_nonzero(d->sensor_mask, N);
        m.nPts = (int)m.sIdx.size();
        m.sW.assign(m.sIdx.size(), 1.0);
    } else if (d->sensor_kind == KW_SENSOR_CARTESIAN && d->sensor_mask) {
        m.haveSampler = true;
        const int nPts = d->sensor_points;
        m.nPts = nPts;
        m.nCorners = 1 << ndim;
        const int nCorners = m.nCorners;
        m.sIdx.resize((size_t)nPts * nCorners);
        m.sW.resize((size_t)nPts * nCorners);
        for (int p = 0; p < nPts; ++p) {
            int i0[3]; double frac[3];
            for (int a = 0; a < ndim; ++a) {
                const double g = (double)d->sensor_mask[(size_t)a * nPts + p] / s.d[a] + (double)(s.n[a] / 2);
                if (!(g >= 0 && g <= (double)(s.n[a] - 1))) { g_err = "Cartesian sensor point outside grid bounds"; return KW_ERR_INVALID; }
                const double f = std::floor(g);
                i0[a] = (int)f; frac[a] = g - f;
            }
            for (int c = 0; c < nCorners; ++c) {
                size_t flat = 0; double w = 1.0;
                for (int a = 0; a < ndim; ++a) {
                    const int bit = (c >> a) & 1;
                    const int ai = std::min(i0[a] + bit, s.n[a] - 1);
                    w *= bit == 1 ? frac[a] : (1.0 - frac[a]);
                    flat = flat * (size_t)s.n[a] + (size_t)ai;
                }
                m.sIdx[(size_t)p * nCorners + c] = flat;
                m.sW[(size_t)p * nCorners + c] = w;
            }
        }
    }

    // 2D directivity (Directivity.swift:41-79): per unique angle, a k-space weight.
    m.directivity = ndim == 2 && d->sensor_kind == KW_SENSOR_BINARY && d->sensor_mask && d->directivity_angle && m.nPts > 0;
    if (m.directivity) {
        std::vector<double> rowAngle(m.nPts);
        for (int r = 0; r < m.nPts; ++r) rowAngle[r] = (double)d->directivity_angle[m.sIdx[r]];
        std::vector<double> uniq(rowAngle);
        std::sort(uniq.begin(), uniq.end());
        uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
        const double elem = std::isnan(d->directivity_size) ? 10.0 * std::max(s.d[0], s.d[1]) : d->directivity_size;
        for (double th : uniq) {
            DirEntry e; e.weight.resize(N);
            for (size_t i = 0; i < N; ++i) {
                const double kx = m.kv[0][s.idx(i, 0)], ky = m.kv[1][s.idx(i, 1)];
                if (d->directivity_pattern == KW_DIRECTIVITY_PRESSURE) {
                    const double kt = std::cos(th) * ky - std::sin(th) * kx;
                    const double x = kt * (elem / 2.0);
                    e.weight[i] = x == 0.0 ? 1.0 : std::sin(M_PI * x) / (M_PI * x);
                } else {
                    const double kn = std::sin(th) * ky + std::cos(th) * kx;
                    e.weight[i] = m.kmag[i] == 0.0 ? 0.0 : kn / m.kmag[i];
                }
            }
            for (int r = 0; r < m.nPts; ++r) if (rowAngle[r] == th) { e.rows.push_back(r); e.gather.push_back(m.sIdx[r]); }
            m.dirEntries.push_back(std::move(e));
        }
    }
    return KW_OK;
}

// SourceOp.apply (KSFO:155-174)
static void apply_source(const Model& m, const SourceOp& op, vecd& field, int t) {
    if (t >= op.len()) return;
    const size_t N = m.N;
    vecd vals(op.idx.size());
    for (size_t q = 0; q < op.idx.size(); ++q)
        vals[q] = (op.signal.size() == 1 ? op.signal[0][t] : op.signal[q][t]) * op.scale[q];
    if (op.mode == KW_SOURCE_DIRICHLET) {
        for (size_t q = 0; q < op.idx.size(); ++q) field[op.idx[q]] = vals[q];
    } else if (op.mode == KW_SOURCE_ADDITIVE_NO_CORRECTION) {
        vecd buf(N, 0.0);
        for (size_t q = 0; q < op.idx.size(); ++q) buf[op.idx[q]] = vals[q];
        for (size_t i = 0; i < N; ++i) field[i] += buf[i];
    } else {
        vecc B(N, cd(0, 0));
        for (size_t q = 0; q < op.idx.size(); ++q) B[op.idx[q]] = vals[q];
        fftn(m.s, B, false);
        for (size_t i = 0; i < N; ++i) B[i] *= m.skappa[i];
        fftn(m.s, B, true);
        for (size_t i = 0; i < N; ++i) field[i] += B[i].real();
    }
}

// One time step t (KSFO:444-521): velocity, sources, density, sources, equation of state, and
// for t = 0 with an initial pressure the override of the whole state.
static void forward_step(const Model& m, State& st, int t, vecc& spec, vecc& work) {
    const Shape& s = m.s;
    const size_t N = m.N;
    const int ndim = m.ndim;
    // velStep (KSFO:448-455): u_a = pml_sg * (pml_sg * u_a - dt/rho_sg * Re ifft(ddPos_a kappa fft(p)))
    spec = to_complex(st.p);
    fftn(s, spec, false);
    for (int a = 0; a < ndim; ++a) {
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)N; ++i) work[i] = m.ddPos[a][s.idx(i, a)] * m.kappa[i] * spec[i];
        fftn(s, work, true);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)N; ++i) {
            const double sg = m.pmlSg[a][s.idx(i, a)];
            st.u[a][i] = sg * (sg * st.u[a][i] - m.dtOverRho[a][i] * work[i].real());
        }
    }
    for (int a = 0; a < ndim; ++a) if (m.hasU[a]) apply_source(m, m.uOp[a], st.u[a], t);   // KSFO:497-501

    // rhoStep (KSFO:457-465): nl factor from the previous split densities
    vecd nl;
    if (m.nonlinear) {
        nl.resize(N);
        for (size_t i = 0; i < N; ++i) {
            double sum = 0;
            for (int a = 0; a < ndim; ++a) sum += st.rho[a][i];
            nl[i] = (2.0 * sum + m.rho0[i]) / m.rho0[i];
        }
    }
    for (int a = 0; a < ndim; ++a) {
        work = to_complex(st.u[a]);
        fftn(s, work, false);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)N; ++i) work[i] *= m.ddNeg[a][s.idx(i, a)] * m.kappa[i];
        fftn(s, work, true);
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < (long long)N; ++i) {
            const double du = work[i].real();
            st.dU[a][i] = du;
            const double mass = m.nonlinear ? m.dtRho0[i] * du * nl[i] : m.dtRho0[i] * du;
            const double pm = m.pml[a][s.idx(i, a)];
            st.rho[a][i] = pm * (pm * st.rho[a][i] - mass);
        }
    }
    for (int a = 0; a < ndim; ++a) if (m.hasP[a]) apply_source(m, m.pOp[a], st.rho[a], t);   // KSFO:503-508

    // eosStep (KSFO:467-474)
    for (size_t i = 0; i < N; ++i) {
        double sum = 0, dsum = 0;
        for (int a = 0; a < ndim; ++a) { sum += st.rho[a][i]; dsum += st.dU[a][i]; }
        st.rhoTot[i] = sum; st.divU[i] = dsum;
    }
    vecd eos(st.rhoTot);
    if (m.absorb) {   // PowerLawAbsorption.eosTerm KSFO:836-845
        if (!m.stokes) {
            for (size_t i = 0; i < N; ++i) work[i] = cd(m.rho0[i] * st.divU[i], 0.0);
            fftn(s, work, false);
            for (size_t i = 0; i < N; ++i) work[i] *= m.nabla1[i];
            fftn(s, work, true);
            for (size_t i = 0; i < N; ++i) eos[i] += m.tau[i] * work[i].real();
        } else {
            for (size_t i = 0; i < N; ++i) eos[i] += m.tau[i] * m.rho0[i] * st.divU[i];
        }
        if (m.dispersion) {
            work = to_complex(st.rhoTot);
            fftn(s, work, false);
            for (size_t i = 0; i < N; ++i) work[i] *= m.nabla2[i];
            fftn(s, work, true);
            for (size_t i = 0; i < N; ++i) eos[i] -= m.eta[i] * work[i].real();
        }
    }
    if (m.nonlinear)
        for (size_t i = 0; i < N; ++i) eos[i] += m.bona[i] * (st.rhoTot[i] * st.rhoTot[i]) / (2.0 * m.rho0[i]);
    for (size_t i = 0; i < N; ++i) st.p[i] = m.c2[i] * eos[i];

    // t = 0 override for an initial pressure (KSFO:514-521; 1D divides by c^2 only, :323)
    if (t == 0 && m.hasP0) {
        st.p = m.p0f;
        for (int a = 0; a < ndim; ++a)
            for (size_t i = 0; i < N; ++i) st.rho[a][i] = ndim == 1 ? m.p0f[i] / m.c2[i] : m.p0f[i] / ((double)ndim * m.c2[i]);
        spec = to_complex(st.p);
        fftn(s, spec, false);
        for (int a = 0; a < ndim; ++a) {
            for (size_t i = 0; i < N; ++i) work[i] = m.ddPos[a][s.idx(i, a)] * m.kappa[i] * spec[i];
            fftn(s, work, true);
            for (size_t i = 0; i < N; ++i) st.u[a][i] = (m.dtOverRho[a][i] / 2.0) * work[i].real();
        }
        for (size_t i = 0; i < N; ++i) {
            double sum = 0;
            for (int a = 0; a < ndim; ++a) sum += st.rho[a][i];
            st.rhoTot[i] = sum;
        }
    }
}

// sensor gather (REC:37-45): binary mask or multilinear Cartesian weights
static void sample_field(const Model& m, const vecd& f, vecd& dst) {
    dst.assign(m.nPts, 0.0);
    for (int p = 0; p < m.nPts; ++p) {
        double acc = 0;
        for (int c = 0; c < m.nCorners; ++c) acc += f[m.sIdx[(size_t)p * m.nCorners + c]] * m.sW[(size_t)p * m.nCorners + c];
        dst[p] = acc;
    }
}

/* ======================================================================================
 * Axisymmetric solver (Solver/KSpaceFirstOrderAS.swift:19-309): x axial (FFT, periodic), y radial
 * (r >= 0). Fields are mirrored into a 4x-expanded radial grid with their symmetry (p, ux: WSWA;
 * uy: HAHS; uy / r: HSHA) and transformed with ordinary 2D FFTs there; the radial PML is
 * one-sided; the divergence gains uy / r on the staggered radial grid r = (j + 1/2) dy.
 * Scope as the reference: p0, pressure and velocity sources (all three modes), Stokes
 * absorption, B/A, p / pFinal recording.
 * ====================================================================================== */
static int run_as(const kw_sim_desc* d, int max_steps, kwref_result** out) {
    if (d->dim != 2) { g_err = "axisymmetric solver requires a 2D grid (x axial, y radial)"; return KW_ERR_INVALID; }
    kw_sim_desc da = *d;
    if (da.alpha_coeff.data && da.alpha_mode != KW_ABSORPTION_NONE) {   // alphaPower ?? 2.0 (:89-93)
        const double y = da.alpha_mode == KW_ABSORPTION_STOKES ? 2.0 : (std::isnan(da.alpha_power) ? 2.0 : da.alpha_power);
        if (std::fabs(y - 2.0) >= 1e-10) { g_err = "axisymmetric absorption requires the Stokes model (alphaPower = 2)"; return KW_ERR_INVALID; }
        da.alpha_mode = KW_ABSORPTION_STOKES;
    }
    d = &da;
    Model m;   // parsing of the medium, sources (signals, scales), p0, sensor (KSFO rules)
    const int st0 = build_model(d, m);
    if (st0 != KW_OK) return st0;
    const int nx = m.s.n[0], ny = m.s.n[1], nyE = 4 * ny;
    const size_t N = m.N, NE = (size_t)nx * nyE;
    const double dx = m.s.d[0], dy = m.s.d[1], dt = m.dt;
    Shape se; se.dim = 2; se.n[0] = nx; se.n[1] = nyE; se.d[0] = dx; se.d[1] = dy; se.finish();
    // k-space operators on the expanded grid (KSpaceFirstOrderAS.swift:51-67)
    const vecd kx = wavenumber_vector(nx, dx), kyE = wavenumber_vector(nyE, dy);
    vecd kappa(NE), skappa(NE);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < nyE; ++j) {
            const double arg = std::sqrt(kx[i] * kx[i] + kyE[j] * kyE[j]) * (m.cRef * dt / 2.0);
            kappa[(size_t)i * nyE + j] = arg == 0.0 ? 1.0 : std::sin(arg) / arg;
            skappa[(size_t)i * nyE + j] = std::cos(arg);
        }
    const cd I(0, 1);
    vecc ddxPos(nx), ddxNeg(nx), ddyPos(nyE), ddyNeg(nyE), yShNeg(nyE);
    for (int i = 0; i < nx; ++i) {
        const double th = kx[i] * dx / 2.0;
        ddxPos[i] = I * kx[i] * cd(std::cos(th), std::sin(th));
        ddxNeg[i] = I * kx[i] * cd(std::cos(th), -std::sin(th));
    }
    for (int j = 0; j < nyE; ++j) {
        const double th = kyE[j] * dy / 2.0;
        ddyPos[j] = I * kyE[j] * cd(std::cos(th), std::sin(th));
        ddyNeg[j] = I * kyE[j] * cd(std::cos(th), -std::sin(th));
        yShNeg[j] = cd(std::cos(th), -std::sin(th));
    }
    // PMLs: axial two-sided, radial outer edge only (PML.swift:17-43 axisymmetric)
    auto one_sided = [&](bool stag) {   // the right ramp of PML.swift:27-41 only
        vecd v(ny, 1.0);
        const double a = d->pml_alpha * (m.cRef / dy), md = (double)d->pml_size;
        for (int k = 0; k < std::min(d->pml_size, ny); ++k) {
            const double x = (double)(k + 1), pos = stag ? (x + 0.5) / md : x / md;
            v[ny - d->pml_size + k] = std::exp(-a * dt / 2.0 * std::pow(pos, 4.0));
        }
        return v;
    };
    const vecd& pmlX = m.pml[0];
    const vecd& pmlXsg = m.pmlSg[0];
    const vecd pmlY = one_sided(false), pmlYsg = one_sided(true);
    vecd invYsg(ny);
    for (int j = 0; j < ny; ++j) invYsg[j] = 1.0 / ((j + 0.5) * dy);
    // pressure source into both density splits with the axial spacing (KSpaceFirstOrderAS.swift:160-163)
    const SourceOp& pOp = m.pOp[0];
    const bool hasP = m.hasP[0];
    const int umode = d->u_mode;

    auto mirror = [&](const vecd& w, int kind, vecc& e) {   // 0 WSWA, 1 HAHS, 2 HSHA
        e.assign(NE, cd(0, 0));
        for (int i = 0; i < nx; ++i) {
            const double* r = &w[(size_t)i * ny];
            cd* o = &e[(size_t)i * nyE];
            if (kind == 0) {
                for (int j = 0; j < ny; ++j) { o[j] = r[j]; o[2 * ny + j] = -r[j]; }
                for (int j = 1; j < ny; ++j) { o[ny + j] = -r[ny - j]; o[3 * ny + j] = r[ny - j]; }
                o[ny] = 0.0; o[3 * ny] = 0.0;
            } else {
                const double sg = kind == 1 ? 1.0 : -1.0;
                for (int j = 0; j < ny; ++j) {
                    o[j] = r[j]; o[ny + j] = sg * r[ny - 1 - j];
                    o[2 * ny + j] = -r[j]; o[3 * ny + j] = -sg * r[ny - 1 - j];
                }
            }
        }
    };
    auto trim = [&](const vecc& e, vecd& w) {
        w.resize(N);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) w[(size_t)i * ny + j] = e[(size_t)i * nyE + j].real();
    };
    vecc E, F2;
    // Re F^-1(H F(mirror(w))) trimmed, H(i, j) on the expanded grid
    auto filtered = [&](const vecd& w, int kind, auto H, vecd& outv) {
        mirror(w, kind, E);
        fftn(se, E, false);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < nyE; ++j) E[(size_t)i * nyE + j] *= H(i, j);
        fftn(se, E, true);
        trim(E, outv);
    };
    auto source_matrix = [&](const SourceOp& op, int t, vecd& mat) {
        mat.assign(N, 0.0);
        for (size_t q = 0; q < op.idx.size(); ++q)
            mat[op.idx[q]] = (op.signal.size() == 1 ? op.signal[0][t] : op.signal[q][t]) * op.scale[q];
    };
    auto apply_u_source = [&](int a, vecd& u, int t, int kind) {
        const SourceOp& op = m.uOp[a];
        if (!m.hasU[a] || t >= op.len()) return;
        vecd mat;
        source_matrix(op, t, mat);
        if (umode == KW_SOURCE_DIRICHLET) {
            for (size_t q = 0; q < op.idx.size(); ++q) u[op.idx[q]] = mat[op.idx[q]];
        } else if (umode == KW_SOURCE_ADDITIVE_NO_CORRECTION) {
            for (size_t i = 0; i < N; ++i) u[i] += mat[i];
        } else {
            vecd c;
            filtered(mat, kind, [&](int i, int j) { return cd(skappa[(size_t)i * nyE + j], 0); }, c);
            for (size_t i = 0; i < N; ++i) u[i] += c[i];
        }
    };
    auto grads = [&](const vecd& p, vecd& gx, vecd& gy) {
        mirror(p, 0, E);
        fftn(se, E, false);
        F2 = E;
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < nyE; ++j) {
                const size_t k = (size_t)i * nyE + j;
                E[k] *= ddxPos[i] * kappa[k];
                F2[k] *= ddyPos[j] * kappa[k];
            }
        fftn(se, E, true);
        fftn(se, F2, true);
        trim(E, gx);
        trim(F2, gy);
    };
    auto sg_rho = [&](int a) {   // dt / rho_sg along axis a (staggerDensity KSFO:799-806)
        const bool map = d->density.len > 1;
        vecd sg = map ? stagger_density(m.s, m.rho0, a) : m.rho0;
        vecd r(N);
        for (size_t i = 0; i < N; ++i) r[i] = dt / sg[i];
        return r;
    };
    const vecd dtorX = sg_rho(0), dtorY = sg_rho(1);

    vecd p(N, 0.0), ux(N, 0.0), uy(N, 0.0), rx(N, 0.0), ry(N, 0.0), gx, gy, duxdx, duydy, t1, t2, mat;
    std::vector<vecd> pRec;
    const int steps = max_steps >= 0 ? std::min(max_steps, m.nt) : m.nt;
    auto tstart = std::chrono::steady_clock::now();
    for (int t = 0; t < steps; ++t) {
        grads(p, gx, gy);
        for (size_t i = 0; i < N; ++i) {
            const int xi = (int)(i / ny), yj = (int)(i % ny);
            ux[i] = pmlXsg[xi] * (pmlXsg[xi] * ux[i] - dtorX[i] * gx[i]);
            uy[i] = pmlYsg[yj] * (pmlYsg[yj] * uy[i] - dtorY[i] * gy[i]);
        }
        apply_u_source(0, ux, t, 0);
        apply_u_source(1, uy, t, 1);
        filtered(ux, 0, [&](int i, int j) { return ddxNeg[i] * kappa[(size_t)i * nyE + j]; }, duxdx);
        {   // duydy = Re F^-1(kappa yShiftNeg (i ky F(HAHS(uy)) + F(HSHA(uy / r))))
            vecd ur(N);
            for (size_t i = 0; i < N; ++i) ur[i] = invYsg[i % ny] * uy[i];
            mirror(uy, 1, E);
            fftn(se, E, false);
            mirror(ur, 2, F2);
            fftn(se, F2, false);
            for (int i = 0; i < nx; ++i)
                for (int j = 0; j < nyE; ++j) {
                    const size_t k = (size_t)i * nyE + j;
                    E[k] = kappa[k] * yShNeg[j] * (I * kyE[j] * E[k] + F2[k]);
                }
            fftn(se, E, true);
            trim(E, duydy);
        }
        for (size_t i = 0; i < N; ++i) {
            const int xi = (int)(i / ny), yj = (int)(i % ny);
            const double dtr = m.nonlinear ? dt * (2.0 * (rx[i] + ry[i]) + m.rho0[i]) : m.dtRho0[i];
            rx[i] = pmlX[xi] * (pmlX[xi] * rx[i] - dtr * duxdx[i]);
            ry[i] = pmlY[yj] * (pmlY[yj] * ry[i] - dtr * duydy[i]);
        }
        if (hasP && t < pOp.len()) {
            source_matrix(pOp, t, mat);
            if (pOp.mode == KW_SOURCE_DIRICHLET) {
                for (size_t q = 0; q < pOp.idx.size(); ++q) { rx[pOp.idx[q]] = mat[pOp.idx[q]]; ry[pOp.idx[q]] = mat[pOp.idx[q]]; }
            } else if (pOp.mode == KW_SOURCE_ADDITIVE_NO_CORRECTION) {
                for (size_t i = 0; i < N; ++i) { rx[i] += mat[i]; ry[i] += mat[i]; }
            } else {
                filtered(mat, 0, [&](int i, int j) { return cd(skappa[(size_t)i * nyE + j], 0); }, t1);
                for (size_t i = 0; i < N; ++i) { rx[i] += t1[i]; ry[i] += t1[i]; }
            }
        }
        for (size_t i = 0; i < N; ++i) {
            const double rt = rx[i] + ry[i];
            double e = rt;
            if (m.absorb) e += m.tau[i] * m.rho0[i] * (duxdx[i] + duydy[i]);
            if (m.nonlinear) e += m.bona[i] * rt * rt / (2.0 * m.rho0[i]);
            p[i] = m.c2[i] * e;
        }
        if (t == 0 && m.hasP0) {
            p = m.p0f;
            for (size_t i = 0; i < N; ++i) { rx[i] = m.p0f[i] / (2.0 * m.c2[i]); ry[i] = rx[i]; }
            grads(p, gx, gy);
            for (size_t i = 0; i < N; ++i) { ux[i] = dtorX[i] / 2.0 * gx[i]; uy[i] = dtorY[i] / 2.0 * gy[i]; }
        }
        if (m.haveSampler && m.recordP) {
            vecd sp;
            sample_field(m, p, sp);
            pRec.push_back(sp);
        }
    }
    auto* R = new kwref_result();
    R->s = m.s; R->nt = m.nt; R->record = d->record; R->steps = steps;
    R->loop_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tstart).count();
    R->fields.assign(KW_FIELD_COUNT, vecd());
    R->present.assign(KW_FIELD_COUNT, 0);
    R->nsensor = m.haveSampler ? m.nPts : 0;
    R->fields[KW_FIELD_P_FINAL] = p;
    R->present[KW_FIELD_P_FINAL] = 1;
    if (!pRec.empty() && (d->record & KW_RECORD_P)) {
        vecd series((size_t)m.nPts * pRec.size());
        for (size_t tt = 0; tt < pRec.size(); ++tt)
            for (int q = 0; q < m.nPts; ++q) series[(size_t)q * pRec.size() + tt] = pRec[tt][q];
        R->fields[KW_FIELD_P] = series;
        R->present[KW_FIELD_P] = 1;
    }
    *out = R;
    return KW_OK;
}

extern "C" {

const char* kwref_last_error(void) { return g_err.c_str(); }

void kwref_free(kwref_result* r) { delete r; }

int kwref_output_size(const kwref_result* r, int field, size_t* count) {
    if (!r || !count || field < 0 || field >= KW_FIELD_COUNT) return KW_ERR_INVALID;
    *count = r->present[field] ? r->fields[field].size() : 0;
    return KW_OK;
}

int kwref_get_output(const kwref_result* r, int field, double* dst, size_t count) {
    if (!r || !dst || field < 0 || field >= KW_FIELD_COUNT) return KW_ERR_INVALID;
    if (!r->present[field] || r->fields[field].size() != count) return KW_ERR_INVALID;
    std::memcpy(dst, r->fields[field].data(), count * sizeof(double));
    return KW_OK;
}

double kwref_loop_seconds(const kwref_result* r) { return r ? r->loop_seconds : 0.0; }
int kwref_steps_done(const kwref_result* r) { return r ? r->steps : 0; }

/* Unit hooks used by the tests. */
int kwref_fft(int n, double* re, double* im, int inverse) {
    FFTPlan pl(n);
    std::vector<cd> x(n);
    for (int i = 0; i < n; ++i) x[i] = cd(re[i], im[i]);
    fft1d(pl, x.data(), inverse != 0);
    for (int i = 0; i < n; ++i) { re[i] = x[i].real(); im[i] = x[i].imag(); }
    return KW_OK;
}

int kwref_pml_profile(int n, double dx, double dt, double c, int m, double alpha, int staggered, double* out) {
    if (m > n || m < 0) return KW_ERR_INVALID;
    vecd v = pml_profile(n, dx, dt, c, m, alpha, staggered != 0);
    std::copy(v.begin(), v.end(), out);
    return KW_OK;
}

int kwref_smooth(int dim, const int* n, const double* in, double* out) {
    Shape s; s.dim = dim;
    for (int a = 0; a < dim; ++a) s.n[a] = n[a];
    s.finish();
    vecd f(in, in + s.N);
    vecd r = smooth_field(s, f);
    std::copy(r.begin(), r.end(), out);
    return KW_OK;
}

int kwref_smoothing_window(int dim, const int* n, double* out) {
    Shape s; s.dim = dim;
    for (int a = 0; a < dim; ++a) s.n[a] = n[a];
    s.finish();
    vecd w = smoothing_window(s);
    std::copy(w.begin(), w.end(), out);
    return KW_OK;
}

double kwref_db2neper(double alpha, double y) { return db2neper(alpha, y); }

/* Run the simulation of `desc` in FP64 (kspaceFirstOrderAS when desc->axisymmetric). max_steps < 0
 * runs all nt steps; otherwise stops after max_steps (used to time a bounded CPU sample).
 * nthreads <= 0 uses every core. */
int kwref_run_timed(const kw_sim_desc* d, int nthreads, int max_steps, int timed_from, kwref_result** out);
int kwref_run(const kw_sim_desc* d, int nthreads, int max_steps, kwref_result** out) {
    return kwref_run_timed(d, nthreads, max_steps, 0, out);
}

/* As kwref_run; kwref_loop_seconds then covers the steps from `timed_from` on (the earlier ones are
 * untimed warm-up steps of a benchmark window). */
int kwref_run_timed(const kw_sim_desc* d, int nthreads, int max_steps, int timed_from, kwref_result** out) {
    if (!d || !out) { g_err = "null argument"; return KW_ERR_INVALID; }
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    if (d->axisymmetric) return run_as(d, max_steps, out);
    Model m;
    const int st0 = build_model(d, m);
    if (st0 != KW_OK) return st0;
    const Shape& s = m.s;
    const size_t N = m.N;
    const int ndim = m.ndim;
    const int nt = m.nt;
    const int nPts = m.nPts;
    const unsigned rec = m.rec;

    auto* R = new kwref_result();
    R->s = s; R->nt = nt; R->record = d->record;
    R->fields.assign(KW_FIELD_COUNT, vecd());
    R->present.assign(KW_FIELD_COUNT, 0);
    R->nsensor = m.haveSampler ? nPts : 0;

    State st;
    st.init(m);
    std::vector<vecd> pRec, uRec[3];
    const int steps = max_steps >= 0 ? std::min(max_steps, nt) : nt;
    auto t0 = std::chrono::steady_clock::now();
    vecc spec(N), work(N);
    for (int t = 0; t < steps; ++t) {
        if (t == timed_from && t > 0) t0 = std::chrono::steady_clock::now();
        forward_step(m, st, t, spec, work);
        // sampling (KSFO:523-540)
        if (m.haveSampler) {
            if (m.recordP) {
                vecd sp;
                if (m.directivity) {
                    sp.assign(nPts, 0.0);
                    vecc P = to_complex(st.p);
                    fftn(s, P, false);
                    for (auto& e : m.dirEntries) {
                        for (size_t i = 0; i < N; ++i) work[i] = P[i] * e.weight[i];
                        fftn(s, work, true);
                        for (size_t q = 0; q < e.rows.size(); ++q) sp[e.rows[q]] = work[e.gather[q]].real();
                    }
                } else {
                    sample_field(m, st.p, sp);
                }
                pRec.push_back(sp);
            }
            if (m.recordU) {
                for (int a = 0; a < ndim; ++a) {
                    work = to_complex(st.u[a]);
                    fftn(s, work, false);
                    for (size_t i = 0; i < N; ++i) work[i] *= m.colloc[a][s.idx(i, a)];
                    fftn(s, work, true);
                    vecd uc(N), su;
                    for (size_t i = 0; i < N; ++i) uc[i] = work[i].real();
                    sample_field(m, uc, su);
                    uRec[a].push_back(su);
                }
            }
        }
    }
    R->loop_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    R->steps = steps;

    // ---- finalizeRecording (REC:129-168) ----
    auto put = [&](int f, vecd v) { R->fields[f] = std::move(v); R->present[f] = 1; };
    put(KW_FIELD_P_FINAL, st.p);
    const int T = steps;
    auto series = [&](const std::vector<vecd>& recs) {   // MLX.stacked(axis: 1) -> [nPts, T]
        vecd v((size_t)nPts * T);
        for (int t = 0; t < T; ++t)
            for (int q = 0; q < nPts; ++q) v[(size_t)q * T + t] = recs[t][q];
        return v;
    };
    const bool haveP = m.haveSampler && m.recordP && T > 0;
    const bool haveU = m.haveSampler && m.recordU && T > 0;
    vecd Pser, User[3];
    if (haveP) Pser = series(pRec);
    if (haveU) for (int a = 0; a < ndim; ++a) User[a] = series(uRec[a]);
    auto reduce_max = [&](const vecd& S) { vecd r(nPts); for (int q = 0; q < nPts; ++q) { double mx = -INFINITY; for (int t = 0; t < T; ++t) mx = std::max(mx, S[(size_t)q * T + t]); r[q] = mx; } return r; };
    auto reduce_min = [&](const vecd& S) { vecd r(nPts); for (int q = 0; q < nPts; ++q) { double mn = INFINITY; for (int t = 0; t < T; ++t) mn = std::min(mn, S[(size_t)q * T + t]); r[q] = mn; } return r; };
    auto reduce_rms = [&](const vecd& S) { vecd r(nPts); for (int q = 0; q < nPts; ++q) { double a = 0; for (int t = 0; t < T; ++t) a += S[(size_t)q * T + t] * S[(size_t)q * T + t]; r[q] = std::sqrt(a / T); } return r; };
    if (haveP) {
        if (rec & KW_RECORD_P) put(KW_FIELD_P, Pser);
        if (rec & KW_RECORD_P_MAX) put(KW_FIELD_P_MAX, reduce_max(Pser));
        if (rec & KW_RECORD_P_MIN) put(KW_FIELD_P_MIN, reduce_min(Pser));
        if (rec & KW_RECORD_P_RMS) put(KW_FIELD_P_RMS, reduce_rms(Pser));
    }
    if (haveU) {
        const unsigned ubits[3] = {KW_RECORD_UX, KW_RECORD_UY, KW_RECORD_UZ};
        for (int a = 0; a < ndim; ++a) {
            if (rec & ubits[a]) put(KW_FIELD_UX + a, User[a]);
            if (rec & KW_RECORD_U_MAX) put(KW_FIELD_UX_MAX + a, reduce_max(User[a]));
            if (rec & KW_RECORD_U_RMS) put(KW_FIELD_UX_RMS + a, reduce_rms(User[a]));
        }
        if ((rec & KW_RECORD_I_AVG) && haveP) {   // intensityAvg REC:113-124
            const int half = T / 2;
            vecc shift(T);
            for (int k = 0; k < T; ++k) {
                const int kk = k <= half ? k : k - T;
                const double th = 2.0 * M_PI * (double)kk / (double)T * 0.5;
                shift[k] = cd(std::cos(th), std::sin(th));
            }
            FFTPlan pl(T);
            for (int a = 0; a < ndim; ++a) {
                vecd r(nPts);
                std::vector<cd> line(T);
                for (int q = 0; q < nPts; ++q) {
                    for (int t = 0; t < T; ++t) line[t] = cd(User[a][(size_t)q * T + t], 0.0);
                    fft1d(pl, line.data(), false);
                    for (int t = 0; t < T; ++t) line[t] *= shift[t];
                    fft1d(pl, line.data(), true);
                    double acc = 0;
                    for (int t = 0; t < T; ++t) acc += Pser[(size_t)q * T + t] * (line[t].real() / T);
                    r[q] = acc / T;
                }
                put(KW_FIELD_IX_AVG + a, r);
            }
        }
    }
    if (m.recordUFinal && (rec & KW_RECORD_U_FINAL))
        for (int a = 0; a < ndim; ++a) put(KW_FIELD_UX_FINAL + a, st.u[a]);
    *out = R;
    return KW_OK;
}

/* ======================================================================================
 * Discrete adjoint (FP64), the reference for the device gradient.
 *
 * L = 1/2 sum_t sum_q (p_q(t) - data_q(t))^2 over the sensor series of forward_step. The
 * reverse sweep transposes every operator of the step in reverse order: the sensor gather, the
 * equation of state (c^2, tau, eta, B/A; the power-law filters |k|^(y-2), |k|^(y-1) are
 * symmetric), the k-space corrected additive pressure source (symmetric cos filter), the PML
 * density update (nl from the previous densities), the staggered derivatives (the transpose of
 * Re F^-1(H F .) is Re F^-1(conj(H) F .)), the PML velocity update, and finally the t = 0
 * override of an initial pressure. Gradients: dL/dc0 (pointwise field), dL/dp0 (the
 * initial pressure after smoothing) and dL/drho0 (pointwise field; a scalar density is treated as
 * a uniform map: the scalar derivative is the sum of the field). rho0 enters the step through
 * dt rho0 (d/drho0 of dt rho0 nl = dt (2 S(t-1) + rho0) is dt), rho0 div in the absorption input,
 * B/A S^2 / (2 rho0), and dt / rho_sg with rho_sg = staggerDensity(rho0) (KSFO:799-806) in the
 * velocity update and the t = 0 override. The whole forward is kept in memory, so this is for small
 * grids. Unsupported (KW_ERR_UNSUPPORTED): velocity sources, Dirichlet or uncorrected pressure
 * sources, directivity, smoothing of c0.
 * ====================================================================================== */
int kwref_adjoint(const kw_sim_desc* d, const double* data, int nthreads, double* misfit, double* grad_c0,
                  double* grad_p0, double* grad_rho0) {
    if (!d || !data) { g_err = "null argument"; return KW_ERR_INVALID; }
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    Model m;
    const int st0 = build_model(d, m);
    if (st0 != KW_OK) return st0;
    for (int a = 0; a < m.ndim; ++a) {
        if (m.hasU[a]) { g_err = "adjoint: velocity sources are not supported"; return KW_ERR_UNSUPPORTED; }
        if (m.hasP[a] && m.pOp[a].mode != KW_SOURCE_ADDITIVE) { g_err = "adjoint: only the k-space corrected additive pressure source is supported"; return KW_ERR_UNSUPPORTED; }
    }
    if (m.directivity) { g_err = "adjoint: directivity is not supported"; return KW_ERR_UNSUPPORTED; }
    if (d->smooth_c0 && d->sound_speed.len > 1) { g_err = "adjoint: smoothC0 is not supported"; return KW_ERR_UNSUPPORTED; }
    if (grad_rho0 && d->smooth_rho0 && d->density.len > 1) { g_err = "adjoint: grad_rho0 with smoothRho0 is not supported"; return KW_ERR_UNSUPPORTED; }
    const bool want_rho = grad_rho0 != nullptr;
    if (!m.haveSampler || m.nPts == 0) { g_err = "adjoint: a sensor is required"; return KW_ERR_INVALID; }
    const Shape& s = m.s;
    const size_t N = m.N;
    const int ndim = m.ndim, nt = m.nt, nPts = m.nPts;

    // ---- forward, keeping what the reverse sweep reads ----
    State st;
    st.init(m);
    std::vector<vecd> P(nt), Ssum(nt), Div(nt), Y(nt);
    std::vector<std::vector<vecd>> DU(nt);
    vecc spec(N), work(N);
    for (int t = 0; t < nt; ++t) {
        forward_step(m, st, t, spec, work);
        P[t] = st.p;
        Ssum[t] = st.rhoTot;
        Div[t] = st.divU;
        if (m.nonlinear || want_rho) DU[t] = st.dU;
        sample_field(m, st.p, Y[t]);
    }
    double L = 0;
    std::vector<vecd> Rs(nt, vecd(nPts));
    for (int t = 0; t < nt; ++t)
        for (int q = 0; q < nPts; ++q) {
            const double r = Y[t][q] - data[(size_t)q * nt + t];
            Rs[t][q] = r;
            L += 0.5 * r * r;
        }
    if (misfit) *misfit = L;

    // ---- reverse sweep ----
    vecd gc(N, 0.0), lp(N, 0.0), tmp, tmp2;
    // dL/drho0 (direct terms) and dL/d(dt / rho_sg_a) per axis
    vecd gr(want_rho ? N : 0, 0.0);
    std::vector<vecd> gdtor(want_rho ? ndim : 0, vecd(N, 0.0));
    // D+_a p (kappa included), the velocity update's derivative of a pressure field
    auto grad_p = [&](const vecd& p, int a, vecd& out) {
        apply_op(m, p, out, [&](size_t i) { return m.ddPos[a][s.idx(i, a)] * m.kappa[i]; });
    };
    std::vector<vecd> lu(ndim, vecd(N, 0.0)), lr(ndim, vecd(N, 0.0));
    const double y = m.y;
    auto scatter_residual = [&](int t) {
        for (int q = 0; q < nPts; ++q)
            for (int c = 0; c < m.nCorners; ++c)
                lp[m.sIdx[(size_t)q * m.nCorners + c]] += m.sW[(size_t)q * m.nCorners + c] * Rs[t][q];
    };
    const int t_stop = m.hasP0 ? 1 : 0;
    for (int t = nt - 1; t >= t_stop; --t) {
        scatter_residual(t);
        const vecd& p = P[t];
        const vecd& S = Ssum[t];
        // equation of state: p = c^2 (S + tau A1(rho0 div) - eta A2(S) + B/A S^2 / (2 rho0))
        vecd q1, q2;
        if (m.absorb && !m.stokes) {
            vecd x(N);
            for (size_t i = 0; i < N; ++i) x[i] = m.rho0[i] * Div[t][i];
            apply_op(m, x, q1, [&](size_t i) { return cd(m.nabla1[i], 0.0); });
        }
        if (m.dispersion) apply_op(m, S, q2, [&](size_t i) { return cd(m.nabla2[i], 0.0); });
        vecd lE(N), lS(N), lDiv(N, 0.0);
        for (size_t i = 0; i < N; ++i) {
            const double c = m.c0[i];
            double dpdc = 2.0 * p[i] / c;
            if (m.absorb) {
                if (m.stokes) dpdc += m.c2[i] * (m.tau[i] / c) * m.rho0[i] * Div[t][i];
                else {
                    dpdc += m.c2[i] * ((y - 1.0) * m.tau[i] / c) * q1[i];
                    if (m.dispersion) dpdc -= m.c2[i] * (y * m.eta[i] / c) * q2[i];
                }
            }
            gc[i] += lp[i] * dpdc;
            lE[i] = m.c2[i] * lp[i];
            lS[i] = lE[i] + (m.nonlinear ? lE[i] * m.bona[i] * S[i] / m.rho0[i] : 0.0);
            // d p / d rho0: B/A S^2 / (2 rho0) and, for Stokes, c^2 tau rho0 div
            if (want_rho) {
                if (m.nonlinear) gr[i] -= lE[i] * m.bona[i] * S[i] * S[i] / (2.0 * m.rho0[i] * m.rho0[i]);
                if (m.absorb && m.stokes) gr[i] += lE[i] * m.tau[i] * Div[t][i];
            }
        }
        if (m.dispersion) {
            vecd x(N);
            for (size_t i = 0; i < N; ++i) x[i] = m.eta[i] * lE[i];
            apply_op(m, x, tmp, [&](size_t i) { return cd(m.nabla2[i], 0.0); });
            for (size_t i = 0; i < N; ++i) lS[i] -= tmp[i];
        }
        if (m.absorb) {
            if (m.stokes) {
                for (size_t i = 0; i < N; ++i) lDiv[i] = m.tau[i] * m.rho0[i] * lE[i];
            } else {
                vecd x(N);
                for (size_t i = 0; i < N; ++i) x[i] = m.tau[i] * lE[i];
                apply_op(m, x, tmp, [&](size_t i) { return cd(m.nabla1[i], 0.0); });
                for (size_t i = 0; i < N; ++i) lDiv[i] = m.rho0[i] * tmp[i];
                // the absorption input rho0 div
                if (want_rho)
                    for (size_t i = 0; i < N; ++i) gr[i] += tmp[i] * Div[t][i];
            }
        }
        // adjoint of the split densities after the source
        std::vector<vecd> Lam(ndim, vecd(N));
        for (int a = 0; a < ndim; ++a)
            for (size_t i = 0; i < N; ++i) Lam[a][i] = lr[a][i] + lS[i];
        // additive source: rho_a += Re F^-1(cos F(buf_a)), buf_a = sig * 2 dt / (d c dx_a) at the mask
        for (int a = 0; a < ndim; ++a) {
            const SourceOp& op = m.pOp[a];
            if (!m.hasP[a] || t >= op.len()) continue;
            apply_op(m, Lam[a], tmp, [&](size_t i) { return cd(m.skappa[i], 0.0); });
            for (size_t q = 0; q < op.idx.size(); ++q) {
                const size_t i = op.idx[q];
                const double sig = op.signal.size() == 1 ? op.signal[0][t] : op.signal[q][t];
                gc[i] += tmp[i] * sig * (-op.scale[q] / m.c0[i]);
            }
        }
        // density update: rho_a = pml_a (pml_a rho_a - dt rho0 nl du_a), nl = (2 S(t-1) + rho0) / rho0
        std::vector<vecd> lDu(ndim, vecd(N));
        vecd lSprev(N, 0.0);
        for (size_t i = 0; i < N; ++i) {
            double nl = 1.0;
            if (m.nonlinear) nl = (2.0 * (t > 0 ? Ssum[t - 1][i] : 0.0) + m.rho0[i]) / m.rho0[i];
            for (int a = 0; a < ndim; ++a) {
                const double pm = m.pml[a][s.idx(i, a)];
                lDu[a][i] = lDiv[i] - pm * m.dtRho0[i] * nl * Lam[a][i];
                if (m.nonlinear) lSprev[i] += -2.0 * m.dt * pm * DU[t][a][i] * Lam[a][i];
                if (want_rho) gr[i] -= pm * m.dt * DU[t][a][i] * Lam[a][i];   // d(dt rho0 nl)/d rho0 = dt
            }
            for (int a = 0; a < ndim; ++a) {
                const double pm = m.pml[a][s.idx(i, a)];
                lr[a][i] = pm * pm * Lam[a][i] + lSprev[i];
            }
        }
        // du_a = D-_a u_a (the new u): mu_a = lambda_u_a + D-_a^T lDu_a
        for (int a = 0; a < ndim; ++a) {
            apply_op(m, lDu[a], tmp, [&](size_t i) { return std::conj(m.ddNeg[a][s.idx(i, a)]) * m.kappa[i]; });
            for (size_t i = 0; i < N; ++i) lu[a][i] += tmp[i];
        }
        // velocity update: u_a = pml_sg (pml_sg u_a - dt/rho_sg D+_a p(t-1))
        vecd lpNew(N, 0.0);
        for (int a = 0; a < ndim; ++a) {
            vecd x(N);
            if (want_rho && t > 0) {   // d u_a / d(dt / rho_sg_a) = -sg D+_a p(t-1); p(-1) = 0
                grad_p(P[t - 1], a, tmp2);
                for (size_t i = 0; i < N; ++i) gdtor[a][i] -= m.pmlSg[a][s.idx(i, a)] * tmp2[i] * lu[a][i];
            }
            for (size_t i = 0; i < N; ++i) {
                const double sg = m.pmlSg[a][s.idx(i, a)];
                x[i] = -sg * m.dtOverRho[a][i] * lu[a][i];
                lu[a][i] = sg * sg * lu[a][i];
            }
            apply_op(m, x, tmp, [&](size_t i) { return std::conj(m.ddPos[a][s.idx(i, a)]) * m.kappa[i]; });
            for (size_t i = 0; i < N; ++i) lpNew[i] += tmp[i];
        }
        lp = lpNew;
    }
    vecd gp(N, 0.0);
    if (m.hasP0) {
        // t = 0 override: p = p0, rho_a = p0 / (d c^2), u_a = dt/rho_sg / 2 D+_a p0
        scatter_residual(0);
        const double dd = ndim == 1 ? 1.0 : (double)ndim;
        for (size_t i = 0; i < N; ++i) {
            double lrs = 0;
            for (int a = 0; a < ndim; ++a) lrs += lr[a][i];
            gp[i] = lp[i] + lrs / (dd * m.c2[i]);
            gc[i] += lrs * m.p0f[i] * (-2.0 / (dd * m.c2[i] * m.c0[i]));
        }
        for (int a = 0; a < ndim; ++a) {
            vecd x(N);
            if (want_rho) {   // u_a = (dt / rho_sg_a) / 2 D+_a p0
                grad_p(m.p0f, a, tmp2);
                for (size_t i = 0; i < N; ++i) gdtor[a][i] += 0.5 * tmp2[i] * lu[a][i];
            }
            for (size_t i = 0; i < N; ++i) x[i] = m.dtOverRho[a][i] / 2.0 * lu[a][i];
            apply_op(m, x, tmp, [&](size_t i) { return std::conj(m.ddPos[a][s.idx(i, a)]) * m.kappa[i]; });
            for (size_t i = 0; i < N; ++i) gp[i] += tmp[i];
        }
    }
    if (grad_c0) for (size_t i = 0; i < N; ++i) grad_c0[i] = gc[i];
    if (grad_p0) for (size_t i = 0; i < N; ++i) grad_p0[i] = gp[i];
    if (want_rho) {
        // dt / rho_sg: d/d rho_sg = -(dt / rho_sg)^2 / dt; rho_sg_a[i] = (rho0[i] + rho0[i + e_a]) / 2,
        // the last index along a replicated (staggerDensity, KSFO:799-806)
        for (int a = 0; a < ndim; ++a) {
            const size_t stride = s.stride[a];
            const int na = s.n[a];
            for (size_t i = 0; i < N; ++i) {
                const double q = m.dtOverRho[a][i];
                const double g = -gdtor[a][i] * q * q / m.dt;
                if (s.idx(i, a) == na - 1) gr[i] += g;
                else { gr[i] += 0.5 * g; gr[i + stride] += 0.5 * g; }
            }
        }
        for (size_t i = 0; i < N; ++i) grad_rho0[i] = gr[i];
    }
    return KW_OK;
}

}  // extern "C"
