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

/* Run the simulation of `desc` in FP64. max_steps < 0 runs all nt steps; otherwise stops
 * after max_steps (used to time a bounded CPU sample). nthreads <= 0 uses every core. */
int kwref_run(const kw_sim_desc* d, int nthreads, int max_steps, kwref_result** out) {
    if (!d || !out) { g_err = "null argument"; return KW_ERR_INVALID; }
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    Shape s;
    s.dim = d->dim;
    if (s.dim < 1 || s.dim > 3) { g_err = "dim must be 1, 2 or 3"; return KW_ERR_INVALID; }
    const int ns[3] = {d->nx, d->ny, d->nz};
    const double ds[3] = {d->dx, d->dy, d->dz};
    for (int a = 0; a < s.dim; ++a) { s.n[a] = ns[a]; s.d[a] = ds[a]; if (ns[a] < 1) { g_err = "bad size"; return KW_ERR_INVALID; } }
    s.finish();
    const size_t N = s.N;
    const int ndim = s.dim;
    const double dt = d->dt;
    const int nt = d->nt;
    if (nt <= 0) { g_err = "call grid.makeTime(...) before running the solver"; return KW_ERR_INVALID; }
    if (!d->p0 && !d->p_mask && !d->u_mask) { g_err = "solver requires source.p0 or a time-varying p/u source"; return KW_ERR_INVALID; }
    if (!grid_sized(d->sound_speed, N) || !grid_sized(d->density, N)) { g_err = "soundSpeed/density must be scalar or grid-shaped"; return KW_ERR_INVALID; }
    if (d->pml_size < 0) { g_err = "bad pml size"; return KW_ERR_INVALID; }
    for (int a = 0; a < ndim; ++a) if (d->pml_size > s.n[a]) { g_err = "pml larger than grid"; return KW_ERR_INVALID; }

    auto* R = new kwref_result();
    R->s = s; R->nt = nt; R->record = d->record;
    R->fields.assign(KW_FIELD_COUNT, vecd());
    R->present.assign(KW_FIELD_COUNT, 0);

    // ---- medium (KSFO:367-373) ----
    const bool c0Map = d->sound_speed.len > 1, rho0Map = d->density.len > 1;
    vecd c0 = expand(d->sound_speed, N), rho0 = expand(d->density, N);
    if (d->smooth_c0 && c0Map) c0 = smooth_field(s, c0);
    if (d->smooth_rho0 && rho0Map) rho0 = smooth_field(s, rho0);
    double cRef = 0;
    for (size_t i = 0; i < N; ++i) cRef = std::max(cRef, c0[i]);   // referenceSoundSpeed KSFO:786-788
    if (!c0Map) cRef = c0[0];
    if (!std::isnan(d->c_ref)) cRef = d->c_ref;

    // ---- k-space operators (KSFO:376-383, 764-769) ----
    std::vector<vecd> kv(ndim);
    for (int a = 0; a < ndim; ++a) kv[a] = wavenumber_vector(s.n[a], s.d[a]);
    vecd kmag(N), kappa(N), skappa(N);
    for (size_t i = 0; i < N; ++i) {
        double k2 = 0;
        for (int a = 0; a < ndim; ++a) { const double k = kv[a][s.idx(i, a)]; k2 += k * k; }
        kmag[i] = std::sqrt(k2);
        const double arg = kmag[i] * (cRef * dt / 2.0);
        kappa[i] = arg == 0.0 ? 1.0 : std::sin(arg) / arg;
        skappa[i] = std::cos(arg);
    }
    std::vector<vecc> ddPos(ndim), ddNeg(ndim), colloc(ndim);
    const cd I(0, 1);
    for (int a = 0; a < ndim; ++a) {
        const int n = s.n[a];
        ddPos[a].resize(n); ddNeg[a].resize(n); colloc[a].resize(n);
        for (int i = 0; i < n; ++i) {
            const double k = kv[a][i], th = k * (s.d[a] / 2.0);
            ddPos[a][i] = I * k * (std::cos(th) + 1.0 * I * std::sin(th));
            ddNeg[a][i] = I * k * (std::cos(th) - 1.0 * I * std::sin(th));
            colloc[a][i] = std::cos(th) - I * std::sin(th);   // REC:101-104
        }
    }

    // ---- PML (KSFO:385-397) ----
    std::vector<vecd> pml(ndim), pmlSg(ndim);
    for (int a = 0; a < ndim; ++a) {
        pml[a] = pml_profile(s.n[a], s.d[a], dt, cRef, d->pml_size, d->pml_alpha, false);
        pmlSg[a] = pml_profile(s.n[a], s.d[a], dt, cRef, d->pml_size, d->pml_alpha, true);
    }

    // ---- staggered density etc. (KSFO:399-402) ----
    vecd c2(N), dtRho0(N);
    for (size_t i = 0; i < N; ++i) { c2[i] = c0[i] * c0[i]; dtRho0[i] = dt * rho0[i]; }
    std::vector<vecd> dtOverRho(ndim);
    for (int a = 0; a < ndim; ++a) {
        vecd sg = rho0Map ? stagger_density(s, rho0, a) : rho0;
        dtOverRho[a].resize(N);
        for (size_t i = 0; i < N; ++i) dtOverRho[a][i] = dt / sg[i];
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
    std::vector<SourceOp> pOp(ndim), uOp(ndim);
    std::vector<bool> hasP(ndim, false), hasU(ndim, false);
    const kw_signal* usig[3] = {&d->ux, &d->uy, &d->uz};
    for (int a = 0; a < ndim; ++a) {
        const int rp = make_op(d->p_mask, d->p, d->p_mode, true, a, pOp[a]);
        const int ru = make_op(d->u_mask, *usig[a], d->u_mode, false, a, uOp[a]);
        if (rp < 0 || ru < 0) { delete R; g_err = "source signal rows must be 1 or the number of source points"; return KW_ERR_INVALID; }
        hasP[a] = rp > 0; hasU[a] = ru > 0;
    }
    auto apply_op = [&](const SourceOp& op, vecd& field, int t) {     // SourceOp.apply KSFO:155-174
        if (t >= op.len()) return;
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
            fftn(s, B, false);
            for (size_t i = 0; i < N; ++i) B[i] *= skappa[i];
            fftn(s, B, true);
            for (size_t i = 0; i < N; ++i) field[i] += B[i].real();
        }
    };

    // ---- p0 (KSFO:425-430) ----
    bool hasP0 = d->p0 != nullptr;
    vecd p0f;
    if (hasP0) {
        p0f.assign(d->p0, d->p0 + N);
        if (d->smooth_p0) p0f = smooth_field(s, p0f);
    }

    // ---- absorption (KSFO:812-882) and nonlinearity (KSFO:889-907) ----
    bool absorb = false, stokes = false, dispersion = false;
    vecd tau, eta, nabla1, nabla2;
    if (d->alpha_coeff.data && d->alpha_mode != KW_ABSORPTION_NONE) {
        if (!grid_sized(d->alpha_coeff, N)) { delete R; g_err = "alphaCoeff must be scalar or grid-shaped"; return KW_ERR_INVALID; }
        absorb = true;
        double y = std::isnan(d->alpha_power) ? 1.5 : d->alpha_power;
        if (d->alpha_mode == KW_ABSORPTION_STOKES) y = 2.0;
        const double np1 = db2neper(1.0, y);
        vecd alphaNp = expand(d->alpha_coeff, N);
        for (auto& v : alphaNp) v *= np1;
        stokes = d->alpha_mode == KW_ABSORPTION_STOKES || std::fabs(y - 2.0) < 1e-10;
        tau.resize(N);
        if (stokes) {
            for (size_t i = 0; i < N; ++i) tau[i] = -2.0 * alphaNp[i] * c0[i];
        } else {
            nabla1.resize(N);
            for (size_t i = 0; i < N; ++i) {
                tau[i] = -2.0 * alphaNp[i] * std::pow(c0[i], y - 1.0);
                nabla1[i] = kmag[i] == 0.0 ? 0.0 : std::pow(kmag[i], y - 2.0);
            }
        }
        if (!stokes && d->alpha_mode != KW_ABSORPTION_NO_DISPERSION) {
            dispersion = true;
            eta.resize(N); nabla2.resize(N);
            const double tn = std::tan(M_PI * y / 2.0);
            for (size_t i = 0; i < N; ++i) {
                eta[i] = 2.0 * alphaNp[i] * std::pow(c0[i], y) * tn;
                nabla2[i] = kmag[i] == 0.0 ? 0.0 : std::pow(kmag[i], y - 1.0);
            }
        }
    }
    bool nonlinear = false;
    vecd bona;
    if (d->b_on_a.data) {
        if (!grid_sized(d->b_on_a, N)) { delete R; g_err = "bOnA must be scalar or grid-shaped"; return KW_ERR_INVALID; }
        bona = expand(d->b_on_a, N);
        double mx = 0;
        for (double v : bona) mx = std::max(mx, std::fabs(v));
        nonlinear = mx != 0.0;
    }

    // ---- sensor (REC:8-97) ----
    const unsigned rec = d->record;
    const bool recordP = (rec & (KW_RECORD_P | KW_RECORD_P_MAX | KW_RECORD_P_MIN | KW_RECORD_P_RMS | KW_RECORD_I_AVG)) != 0;
    const bool recordU = (rec & (KW_RECORD_UX | KW_RECORD_UY | KW_RECORD_UZ | KW_RECORD_U_MAX | KW_RECORD_U_RMS | KW_RECORD_I_AVG)) != 0;
    const bool recordUFinal = (rec & KW_RECORD_U_FINAL) != 0;
    bool haveSampler = false;
    int nPts = 0, nCorners = 1;
    std::vector<size_t> sIdx;
    vecd sW;
    if (d->sensor_kind == KW_SENSOR_BINARY && d->sensor_mask) {
        haveSampler = true;
        sIdx = flat_nonzero(d->sensor_mask, N);
        nPts = (int)sIdx.size();
        sW.assign(sIdx.size(), 1.0);
    } else if (d->sensor_kind == KW_SENSOR_CARTESIAN && d->sensor_mask) {
        haveSampler = true;
        nPts = d->sensor_points;
        nCorners = 1 << ndim;
        sIdx.resize((size_t)nPts * nCorners);
        sW.resize((size_t)nPts * nCorners);
        for (int p = 0; p < nPts; ++p) {
            int i0[3]; double frac[3];
            for (int a = 0; a < ndim; ++a) {
                const double g = (double)d->sensor_mask[(size_t)a * nPts + p] / s.d[a] + (double)(s.n[a] / 2);
                if (!(g >= 0 && g <= (double)(s.n[a] - 1))) { delete R; g_err = "Cartesian sensor point outside grid bounds"; return KW_ERR_INVALID; }
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
                sIdx[(size_t)p * nCorners + c] = flat;
                sW[(size_t)p * nCorners + c] = w;
            }
        }
    }
    R->nsensor = haveSampler ? nPts : 0;

    // 2D directivity (Directivity.swift:41-79): per unique angle, a k-space weight.
    struct DirEntry { vecd weight; std::vector<int> rows; std::vector<size_t> gather; };
    std::vector<DirEntry> dirEntries;
    const bool directivity = ndim == 2 && d->sensor_kind == KW_SENSOR_BINARY && d->sensor_mask && d->directivity_angle && nPts > 0;
    if (directivity) {
        std::vector<double> rowAngle(nPts);
        for (int r = 0; r < nPts; ++r) rowAngle[r] = (double)d->directivity_angle[sIdx[r]];
        std::vector<double> uniq(rowAngle);
        std::sort(uniq.begin(), uniq.end());
        uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
        const double elem = std::isnan(d->directivity_size) ? 10.0 * std::max(s.d[0], s.d[1]) : d->directivity_size;
        for (double th : uniq) {
            DirEntry e; e.weight.resize(N);
            for (size_t i = 0; i < N; ++i) {
                const double kx = kv[0][s.idx(i, 0)], ky = kv[1][s.idx(i, 1)];
                if (d->directivity_pattern == KW_DIRECTIVITY_PRESSURE) {
                    const double kt = std::cos(th) * ky - std::sin(th) * kx;
                    const double x = kt * (elem / 2.0);
                    e.weight[i] = x == 0.0 ? 1.0 : std::sin(M_PI * x) / (M_PI * x);
                } else {
                    const double kn = std::sin(th) * ky + std::cos(th) * kx;
                    e.weight[i] = kmag[i] == 0.0 ? 0.0 : kn / kmag[i];
                }
            }
            for (int r = 0; r < nPts; ++r) if (rowAngle[r] == th) { e.rows.push_back(r); e.gather.push_back(sIdx[r]); }
            dirEntries.push_back(std::move(e));
        }
    }

    auto sample = [&](const vecd& f, vecd& dst) {
        dst.assign(nPts, 0.0);
        for (int p = 0; p < nPts; ++p) {
            double acc = 0;
            for (int c = 0; c < nCorners; ++c) acc += f[sIdx[(size_t)p * nCorners + c]] * sW[(size_t)p * nCorners + c];
            dst[p] = acc;
        }
    };

    // ---- state (KSFO:438-442) ----
    vecd p(N, 0.0), rhoTot(N), divU(N);
    std::vector<vecd> u(ndim, vecd(N, 0.0)), rho(ndim, vecd(N, 0.0)), dU(ndim, vecd(N, 0.0));
    std::vector<vecd> pRec, uRec[3];

    const int steps = max_steps >= 0 ? std::min(max_steps, nt) : nt;
    auto t0 = std::chrono::steady_clock::now();
    vecc spec(N), work(N);
    for (int t = 0; t < steps; ++t) {
        // velStep (KSFO:448-455): u_a = pml_sg * (pml_sg * u_a - dt/rho_sg * Re ifft(ddPos_a kappa fft(p)))
        spec = to_complex(p);
        fftn(s, spec, false);
        for (int a = 0; a < ndim; ++a) {
#pragma omp parallel for schedule(static)
            for (long long i = 0; i < (long long)N; ++i) work[i] = ddPos[a][s.idx(i, a)] * kappa[i] * spec[i];
            fftn(s, work, true);
#pragma omp parallel for schedule(static)
            for (long long i = 0; i < (long long)N; ++i) {
                const double sg = pmlSg[a][s.idx(i, a)];
                u[a][i] = sg * (sg * u[a][i] - dtOverRho[a][i] * work[i].real());
            }
        }
        for (int a = 0; a < ndim; ++a) if (hasU[a]) apply_op(uOp[a], u[a], t);   // KSFO:497-501

        // rhoStep (KSFO:457-465): nl factor from the previous split densities
        vecd nl;
        if (nonlinear) {
            nl.resize(N);
            for (size_t i = 0; i < N; ++i) {
                double sum = 0;
                for (int a = 0; a < ndim; ++a) sum += rho[a][i];
                nl[i] = (2.0 * sum + rho0[i]) / rho0[i];
            }
        }
        for (int a = 0; a < ndim; ++a) {
            work = to_complex(u[a]);
            fftn(s, work, false);
#pragma omp parallel for schedule(static)
            for (long long i = 0; i < (long long)N; ++i) work[i] *= ddNeg[a][s.idx(i, a)] * kappa[i];
            fftn(s, work, true);
#pragma omp parallel for schedule(static)
            for (long long i = 0; i < (long long)N; ++i) {
                const double du = work[i].real();
                dU[a][i] = du;
                const double mass = nonlinear ? dtRho0[i] * du * nl[i] : dtRho0[i] * du;
                const double pm = pml[a][s.idx(i, a)];
                rho[a][i] = pm * (pm * rho[a][i] - mass);
            }
        }
        for (int a = 0; a < ndim; ++a) if (hasP[a]) apply_op(pOp[a], rho[a], t);   // KSFO:503-508

        // eosStep (KSFO:467-474)
        for (size_t i = 0; i < N; ++i) {
            double sum = 0, dsum = 0;
            for (int a = 0; a < ndim; ++a) { sum += rho[a][i]; dsum += dU[a][i]; }
            rhoTot[i] = sum; divU[i] = dsum;
        }
        vecd eos(rhoTot);
        if (absorb) {   // PowerLawAbsorption.eosTerm KSFO:836-845
            if (!stokes) {
                for (size_t i = 0; i < N; ++i) work[i] = cd(rho0[i] * divU[i], 0.0);
                fftn(s, work, false);
                for (size_t i = 0; i < N; ++i) work[i] *= nabla1[i];
                fftn(s, work, true);
                for (size_t i = 0; i < N; ++i) eos[i] += tau[i] * work[i].real();
            } else {
                for (size_t i = 0; i < N; ++i) eos[i] += tau[i] * rho0[i] * divU[i];
            }
            if (dispersion) {
                work = to_complex(rhoTot);
                fftn(s, work, false);
                for (size_t i = 0; i < N; ++i) work[i] *= nabla2[i];
                fftn(s, work, true);
                for (size_t i = 0; i < N; ++i) eos[i] -= eta[i] * work[i].real();
            }
        }
        if (nonlinear)
            for (size_t i = 0; i < N; ++i) eos[i] += bona[i] * (rhoTot[i] * rhoTot[i]) / (2.0 * rho0[i]);
        for (size_t i = 0; i < N; ++i) p[i] = c2[i] * eos[i];

        // t = 0 override for an initial pressure (KSFO:514-521; 1D divides by c^2 only, :323)
        if (t == 0 && hasP0) {
            p = p0f;
            for (int a = 0; a < ndim; ++a)
                for (size_t i = 0; i < N; ++i) rho[a][i] = ndim == 1 ? p0f[i] / c2[i] : p0f[i] / ((double)ndim * c2[i]);
            spec = to_complex(p);
            fftn(s, spec, false);
            for (int a = 0; a < ndim; ++a) {
                for (size_t i = 0; i < N; ++i) work[i] = ddPos[a][s.idx(i, a)] * kappa[i] * spec[i];
                fftn(s, work, true);
                for (size_t i = 0; i < N; ++i) u[a][i] = (dtOverRho[a][i] / 2.0) * work[i].real();
            }
        }

        // sampling (KSFO:523-540)
        if (haveSampler) {
            if (recordP) {
                vecd sp;
                if (directivity) {
                    sp.assign(nPts, 0.0);
                    vecc P = to_complex(p);
                    fftn(s, P, false);
                    for (auto& e : dirEntries) {
                        for (size_t i = 0; i < N; ++i) work[i] = P[i] * e.weight[i];
                        fftn(s, work, true);
                        for (size_t q = 0; q < e.rows.size(); ++q) sp[e.rows[q]] = work[e.gather[q]].real();
                    }
                } else {
                    sample(p, sp);
                }
                pRec.push_back(sp);
            }
            if (recordU) {
                for (int a = 0; a < ndim; ++a) {
                    work = to_complex(u[a]);
                    fftn(s, work, false);
                    for (size_t i = 0; i < N; ++i) work[i] *= colloc[a][s.idx(i, a)];
                    fftn(s, work, true);
                    vecd uc(N), su;
                    for (size_t i = 0; i < N; ++i) uc[i] = work[i].real();
                    sample(uc, su);
                    uRec[a].push_back(su);
                }
            }
        }
    }
    R->loop_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    R->steps = steps;

    // ---- finalizeRecording (REC:129-168) ----
    auto put = [&](int f, vecd v) { R->fields[f] = std::move(v); R->present[f] = 1; };
    put(KW_FIELD_P_FINAL, p);
    const int T = steps;
    auto series = [&](const std::vector<vecd>& recs) {   // MLX.stacked(axis: 1) -> [nPts, T]
        vecd v((size_t)nPts * T);
        for (int t = 0; t < T; ++t)
            for (int q = 0; q < nPts; ++q) v[(size_t)q * T + t] = recs[t][q];
        return v;
    };
    const bool haveP = haveSampler && recordP && T > 0;
    const bool haveU = haveSampler && recordU && T > 0;
    vecd Pser, User[3];
    if (haveP) Pser = series(pRec);
    if (haveU) for (int a = 0; a < ndim; ++a) User[a] = series(uRec[a]);
    auto reduce_max = [&](const vecd& S) { vecd r(nPts); for (int q = 0; q < nPts; ++q) { double m = -INFINITY; for (int t = 0; t < T; ++t) m = std::max(m, S[(size_t)q * T + t]); r[q] = m; } return r; };
    auto reduce_min = [&](const vecd& S) { vecd r(nPts); for (int q = 0; q < nPts; ++q) { double m = INFINITY; for (int t = 0; t < T; ++t) m = std::min(m, S[(size_t)q * T + t]); r[q] = m; } return r; };
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
    if (recordUFinal && (rec & KW_RECORD_U_FINAL))
        for (int a = 0; a < ndim; ++a) put(KW_FIELD_UX_FINAL + a, u[a]);
    *out = R;
    return KW_OK;
}

}  // extern "C"
