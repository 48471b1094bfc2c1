// kw_engine.cpp — host side of the solver: validation, FP64 precompute, device buffers, the
// per-step launch sequence (captured as a CUDA graph), recording and output copy-out.
//
// Reference: k-wave-swift Sources/KWave/Solver/KSpaceFirstOrder.swift (KSFO) and
// Sources/KWave/Sensor/Recording.swift (REC). The per-step order of operations follows
// KSFO:492-546: velocity update, velocity sources, density update, pressure sources, equation of
// state, t = 0 initial-pressure override, sensor sampling.
#include "kw_engine.h"
#include "kw_host.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>

namespace kw {

static constexpr size_t kSmemBudget = 100 * 1024;  // per CTA: two CTAs per SM

static KwError err(int code, const std::string& m) { return KwError{code, m}; }

void Engine::check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw err(KW_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

void* Engine::dalloc(size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (fail_alloc_ > 0 && ++nalloc_ == fail_alloc_)
        throw err(KW_ERR_OOM, "device allocation of " + std::to_string(bytes) +
                                  " bytes failed (KW_TEST_FAIL_ALLOC: simulated out-of-memory)");
    if (arena_) {
        // allocation-free mode: carve 256-byte aligned pieces out of the caller-provided region
        const size_t off = (arena_used_ + 255) & ~(size_t)255;
        if (off + bytes > arena_size_)
            throw err(KW_ERR_INVALID, "problem needs more than the " + std::to_string(arena_size_) +
                                          "-byte allocation-free scratch (at least " + std::to_string(off + bytes) +
                                          " bytes); use the allocating entry point");
        arena_used_ = off + bytes;
        check(cudaMemsetAsync(arena_ + off, 0, bytes, st()), "memset");
        return arena_ + off;
    }
    const size_t rounded = Context::round_block(bytes);
    void* p = ctx_->cache_take(rounded);
    if (!p) {
        cudaError_t e = cudaMalloc(&p, rounded);
        if (e != cudaSuccess) {   // blocks kept for later creates may be what is missing
            cudaGetLastError();
            ctx_->cache_release();
            e = cudaMalloc(&p, rounded);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw err(KW_ERR_OOM, "device allocation of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
        }
    }
    allocs_.emplace_back(p, rounded);
    check(cudaMemsetAsync(p, 0, bytes, st()), "memset");
    return p;
}

void* Context::cache_take(size_t rounded) {
    std::lock_guard<std::mutex> lock(cache_mu);
    auto it = cache.find(rounded);
    if (it == cache.end()) return nullptr;
    void* p = it->second;
    cache.erase(it);
    cached_bytes -= rounded;
    return p;
}

void Context::cache_put(void* p, size_t rounded) {
    std::lock_guard<std::mutex> lock(cache_mu);
    if (!cache_cap) {   // a quarter of the device's memory
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            cudaGetLastError();
            total_b = 0;
        }
        cache_cap = total_b ? total_b / 4 : (size_t)1 << 30;
    }
    if (cached_bytes + rounded > cache_cap) {   // over the cap: give the block back
        cudaFree(p);
        return;
    }
    cache.emplace(rounded, p);
    cached_bytes += rounded;
}

void Context::cache_release() {
    std::lock_guard<std::mutex> lock(cache_mu);
    for (auto& kv : cache) cudaFree(kv.second);
    cache.clear();
    cached_bytes = 0;
}

Context::~Context() {
    cache_release();
    for (int b = 0; b < 2; ++b) {
        if (stage_ev[b]) {
            cudaEventSynchronize(stage_ev[b]);
            cudaEventDestroy(stage_ev[b]);
        }
        if (stage[b]) cudaFreeHost(stage[b]);
    }
}

// device -> host copy into a caller's (pageable) buffer, staged through the context's pinned
// buffers when it is large: the DMA of chunk k + 1 runs while the host threads copy chunk k out
// of the other buffer. Returns when the data are in `dst`.
void Engine::download_host(void* dst, const void* src, size_t bytes) {
    constexpr size_t kSub = 1u << 20;
    Context& c = *ctx_;
    std::unique_lock<std::mutex> lock(c.stage_mu);
    if (bytes < 2 * kSub || !stage_ready_locked()) {
        lock.unlock();
        check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st()), "output copy");
        check(cudaStreamSynchronize(st()), "output copy");
        return;
    }
    const char* s = static_cast<const char*>(src);
    char* d = static_cast<char*>(dst);
    const size_t nchunk = (bytes + Context::kStageBytes - 1) / Context::kStageBytes;
    auto host_copy = [&](size_t k) {   // chunk k from its buffer to the caller's
        const int b = (int)(k & 1);
        check(cudaEventSynchronize(c.stage_ev[b]), "stage wait");
        const size_t off = k * Context::kStageBytes, len = std::min(Context::kStageBytes, bytes - off);
        const char* buf = static_cast<const char*>(c.stage[b]);
        parallel_for((long long)((len + kSub - 1) / kSub), [&](long long q) {
            const size_t lo = (size_t)q * kSub, n = std::min(kSub, len - lo);
            std::memcpy(d + off + lo, buf + lo, n);
        }, 2);
    };
    for (size_t k = 0; k < nchunk; ++k) {
        const int b = (int)(k & 1);
        const size_t off = k * Context::kStageBytes, len = std::min(Context::kStageBytes, bytes - off);
        check(cudaEventSynchronize(c.stage_ev[b]), "stage wait");   // its previous copy is finished
        check(cudaMemcpyAsync(c.stage[b], s + off, len, cudaMemcpyDeviceToHost, st()), "output copy");
        check(cudaEventRecord(c.stage_ev[b], st()), "stage event");
        if (k > 0) host_copy(k - 1);
    }
    host_copy(nchunk - 1);
}

// the two pinned staging buffers and their events, allocated on first use (false: no pinned memory)
bool Engine::stage_ready_locked() {
    Context& c = *ctx_;
    if (c.stage[0] && c.stage[1]) return true;
    if (c.stage_failed) return false;
    bool ok = true;
    for (int b = 0; b < 2 && ok; ++b)
        ok = cudaHostAlloc(&c.stage[b], Context::kStageBytes, cudaHostAllocDefault) == cudaSuccess &&
             cudaEventCreateWithFlags(&c.stage_ev[b], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {   // plain copies from then on
        cudaGetLastError();
        for (int b = 0; b < 2; ++b) {
            if (c.stage[b]) cudaFreeHost(c.stage[b]);
            if (c.stage_ev[b]) cudaEventDestroy(c.stage_ev[b]);
            c.stage[b] = nullptr;
            c.stage_ev[b] = nullptr;
        }
        c.stage_failed = true;
    }
    return ok;
}

void Engine::upload_host(void* dst, const void* src, size_t bytes) {
    constexpr size_t kSub = 1u << 20;   // one host thread copies 1 MiB pieces of a chunk
    Context& c = *ctx_;
    std::unique_lock<std::mutex> lock(c.stage_mu);
    if (bytes < 2 * kSub || !stage_ready_locked()) {
        lock.unlock();
        check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st()), "upload");
        return;
    }
    const char* s = static_cast<const char*>(src);
    char* d = static_cast<char*>(dst);
    for (size_t off = 0, k = 0; off < bytes; off += Context::kStageBytes, ++k) {
        const int b = (int)(k & 1);
        check(cudaEventSynchronize(c.stage_ev[b]), "stage wait");   // the buffer's previous copy is done
        const size_t len = std::min(Context::kStageBytes, bytes - off);
        char* buf = static_cast<char*>(c.stage[b]);
        parallel_for((long long)((len + kSub - 1) / kSub), [&](long long q) {
            const size_t lo = (size_t)q * kSub, n = std::min(kSub, len - lo);
            std::memcpy(buf + lo, s + off + lo, n);
        }, 2);
        check(cudaMemcpyAsync(d + off, buf, len, cudaMemcpyHostToDevice, st()), "upload");
        check(cudaEventRecord(c.stage_ev[b], st()), "stage event");
    }
}

Engine::~Engine() {
    if (poll_ev_) cudaEventDestroy(poll_ev_);
    if (poll_host_) cudaFreeHost(poll_host_);
    for (int v = 0; v < 2; ++v) {
        if (graph_exec_[v]) cudaGraphExecDestroy(graph_exec_[v]);
        if (graph_[v]) cudaGraphDestroy(graph_[v]);
    }
    cudaStreamSynchronize(ctx_->stream);
    if (cudaGetLastError() == cudaSuccess && !arena_)
        for (auto& a : allocs_) ctx_->cache_put(a.first, a.second);   // kept for the next create
    else
        for (auto& a : allocs_) cudaFree(a.first);
}

// ------------------------------------------------------------------------------------------
// FP64 helpers (restated from the reference's host setup)
// ------------------------------------------------------------------------------------------

// 2 pi fftfreq(n, d)   (Internal/Support.swift:6-19)
static std::vector<double> wavenumbers(int n, double d) {
    std::vector<double> r(n);
    const double val = 1.0 / ((double)n * d);
    const int cutoff = (n - 1) / 2 + 1;
    for (int i = 0; i < cutoff; ++i) r[i] = (double)i * val;
    int j = -(n / 2);
    for (int i = cutoff; i < n; ++i) r[i] = (double)(j++) * val;
    for (auto& v : r) v *= 2.0 * M_PI;
    return r;
}

// pmlProfile (PML/PML.swift:17-43)
static std::vector<double> pml_profile(int n, double dx, double dt, double c, int m, double alpha, bool staggered) {
    const double a = alpha * (c / dx);
    const double md = (double)m;
    std::vector<double> pml(n, 1.0);
    for (int k = 0; k < std::min(m, n); ++k) {
        const double x = (double)(k + 1);
        const double pl = staggered ? (md + 0.5 - x) / md : (md + 1.0 - x) / md;
        const double pr = staggered ? (x + 0.5) / md : x / md;
        pml[k] = std::exp(-a * dt / 2.0 * std::pow(pl, 4.0));
        pml[n - m + k] = std::exp(-a * dt / 2.0 * std::pow(pr, 4.0));
    }
    return pml;
}

static double db2neper(double alpha, double y) {  // Material/Conversion.swift:6-8
    return 100.0 * alpha * std::pow(1e-6 / (2.0 * M_PI), y) / (20.0 * std::log10(M_E));
}

static std::vector<float> to_f32(const std::vector<double>& v) {
    std::vector<float> r(v.size());
    for (size_t i = 0; i < v.size(); ++i) r[i] = (float)v[i];
    return r;
}

// ------------------------------------------------------------------------------------------
// FFT plans: Stockham radix sequence + FP64 twiddles rounded to FP32
// ------------------------------------------------------------------------------------------
void Engine::build_plan(FFTPlanDev& pl, int n) {
    std::memset(&pl, 0, sizeof(pl));
    pl.n = n;
    std::vector<int> rad;
    int m = n;
    for (int r : {16, 8, 4, 2, 3, 5}) {
        while (m % r == 0) { rad.push_back(r); m /= r; }
    }
    for (int p = 7; m > 1; p += 2) {
        while (m % p == 0) { rad.push_back(p); m /= p; }
        if ((long long)p * p > m && m > 1) { rad.push_back(m); m = 1; }
    }
    if ((int)rad.size() > kMaxStages) throw err(KW_ERR_UNSUPPORTED, "FFT length " + std::to_string(n) + " has too many factors");
    for (int r : rad)
        if (r > 64) throw err(KW_ERR_UNSUPPORTED, "FFT length " + std::to_string(n) + " has a prime factor above 64");
    pl.nstages = (int)rad.size();
    std::vector<float2> tw, gen;
    int Ns = 1;
    for (int s = 0; s < pl.nstages; ++s) {
        const int R = rad[s];
        pl.radix[s] = R;
        pl.tw_off[s] = (int)tw.size();
        for (int k = 0; k < Ns; ++k)
            for (int r = 1; r < R; ++r) {
                const double a = -2.0 * M_PI * (double)r * (double)k / (double)(Ns * R);
                tw.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
            }
        pl.gen_off[s] = (int)gen.size();
        if (R != 2 && R != 3 && R != 4 && R != 5 && R != 8 && R != 16)
            for (int q = 0; q < R; ++q) {
                const double a = -2.0 * M_PI * (double)q / (double)R;
                gen.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
            }
        Ns *= R;
    }
    if (tw.empty()) tw.push_back(make_float2(1.f, 0.f));
    if (gen.empty()) gen.push_back(make_float2(1.f, 0.f));
    pl.tw = upload(tw);
    pl.gen = upload(gen);
    std::vector<float2> twn(std::max(n, 1));
    for (int m2 = 0; m2 < n; ++m2) {
        const double a = -2.0 * M_PI * (double)m2 / (double)n;
        twn[m2] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    pl.twn = upload(twn);
}

// ------------------------------------------------------------------------------------------
// one time step (KSFO:492-546)
// ------------------------------------------------------------------------------------------
void Engine::issue_step(bool first) {
    if (as_mode_) {
        issue_step_as(first);
        return;
    }
    const int D = dim_;
    const int sp1 = D == 1 ? 0 : 1;   // first output spectrum
    // row fusion (kw_jobs.cpp): the velocity C2R transforms the new u_a into the density job's
    // spectra unless a velocity source changes u in between; the density C2R transforms
    // rho0 div u and rho_sum into the absorption job's spectra unless a pressure source job or a
    // Dirichlet source changes them in between (and not while the adjoint tape is recorded)
    const bool fuse = D >= 2 && fuse_rows();
    const bool fuse_vel = fuse && !any_u_direct_ && !any_u_add_;
    const bool fuse_den = fuse && any_abs_ && !tape_mode_ && !any_p_direct_ && !any_p_add_;

    // velocity update: u_a = pml_sg (pml_sg u_a - dt/rho_sg Re F^-1(ddPos_a kappa F(p)))
    SpecJob vel;
    vel.in_field = FS_P;
    vel.nin = 1;
    vel.fanout = 1;
    vel.nout = D;
    for (int a = 0; a < D; ++a) vel.op[a] = OpSpec{AO_DPOS, (int8_t)a, RT_KAPPA, 0};
    vel.spec_in = 0;
    vel.spec_out = sp1;
    vel.epi = EPI_VEL;
    vel.fwd_spec = fuse_vel ? sp1 : -1;   // the density job's input spectra
    vel.name = "vel";
    issue_job(vel, -1);

    // velocity sources
    if (any_u_direct_) timed("src_u", 0, [&] { launch_src_u(st(), d_sims_, d_t_, count(), max_usrc_, 0); });
    if (any_u_add_) {
        timed("src_u_scatter", 0, [&] { launch_src_u(st(), d_sims_, d_t_, count(), max_usrc_, 1); });
        SpecJob us;
        us.in_field = FS_SRCBUF;
        us.nin = D;
        us.nout = D;
        for (int a = 0; a < D; ++a) us.op[a] = OpSpec{AO_NONE, (int8_t)a, RT_SKAPPA, (int8_t)a};
        us.spec_in = sp1;
        us.spec_out = sp1;
        us.epi = EPI_ADD_U;
        us.gate = GATE_USRC;
        us.name = "usrc";
        issue_job(us, -1);
    }

    // density update + (pointwise) equation of state
    SpecJob den;
    den.in_field = FS_U;
    den.nin = D;
    den.nout = D;
    for (int a = 0; a < D; ++a) den.op[a] = OpSpec{AO_DNEG, (int8_t)a, RT_KAPPA, (int8_t)a};
    den.spec_in = sp1;
    den.spec_out = sp1;
    den.epi = psrc_live() ? EPI_DEN_SRC : EPI_DEN;
    den.tape = tape_mode_ ? 1 : 0;
    den.coupled = 1;
    den.r2c_done = fuse_vel ? 1 : 0;
    den.fwd_spec = fuse_den ? 0 : -1;   // the absorption job's input spectra
    den.name = "den";
    issue_job(den, -1);

    // pressure sources
    if (any_p_direct_) timed("src_p", 0, [&] { launch_src_p(st(), d_sims_, d_t_, count(), max_psrc_, 0); });
    if (any_p_add_) {
        timed("src_p_scatter", 0, [&] { launch_src_p(st(), d_sims_, d_t_, count(), max_psrc_, 1); });
        SpecJob ps;
        ps.in_field = FS_SRCBUF;
        ps.nin = 1;
        ps.nout = 1;
        ps.op[0] = OpSpec{AO_NONE, 0, RT_SKAPPA, 0};
        ps.spec_in = 0;
        ps.spec_out = 0;
        ps.epi = EPI_ADD_RHO;
        ps.tape = tape_mode_ ? 1 : 0;
        ps.gate = GATE_PSRC;
        ps.name = "psrc";
        issue_job(ps, -1);
    }

    // power-law absorption and dispersion, then the equation of state
    if (any_abs_) {
        SpecJob ab;
        ab.in_field = FS_WORK;   // comp 0: rho0 * div u, comp 1: rho_sum
        ab.nin = 2;
        ab.nout = 2;
        ab.op[0] = OpSpec{AO_NONE, 0, RT_NU1, 0};
        ab.op[1] = OpSpec{AO_NONE, 0, RT_NU2, 1};
        ab.spec_in = 0;
        ab.spec_out = 0;
        ab.epi = EPI_EOS_ABS;
        ab.tape = tape_mode_ ? 1 : 0;
        ab.coupled = 1;
        ab.gate = GATE_ABS;
        ab.r2c_done = fuse_den ? 1 : 0;
        ab.name = "abs";
        issue_job(ab, -1);
    }

    // t = 0 override for an initial pressure (KSFO:514-521)
    if (first && any_p0_) {
        const Map& m = map_elems(-1);
        launch_init_p0(st(), d_sims_, d_t_, m.d, m.n, d_p0s_);
        SpecJob vi = vel;
        vi.epi = EPI_VEL_INIT;
        vi.fwd_spec = -1;
        vi.gate = GATE_P0;
        vi.name = "vel0";
        issue_job(vi, -1);
    }

    // sensor sampling (KSFO:523-540); 2D directivity first filters p once per angle
    // (Directivity.swift:41-79)
    if (any_recp_)
        for (int j = 0; j < max_dir_; ++j) {
            SpecJob dj;
            dj.in_field = FS_P;
            dj.nin = 1;
            dj.nout = 1;
            dj.op[0] = OpSpec{AO_NONE, 0, (int8_t)(RT_DIR0 + j), 0};
            dj.spec_in = 0;
            dj.spec_out = 0;
            dj.epi = EPI_STORE;
            dj.out_field = FS_DIR + j;
            dj.gate = GATE_DIR + j;
            dj.name = "dir";
            issue_job(dj, -1);
        }
    // the pressure sample, when it is the step's last launch, also advances the step counter
    const bool tick_in_sample = any_recp_ && !any_recu_ && max_pts_ > 0;
    if (any_recp_)
        timed("sample_p", 0, [&] {
            launch_sample(st(), d_sims_, d_t_, count(), max_pts_, 0, 0, tick_in_sample ? d_tickc_ : nullptr);
        });
    if (any_recu_) {
        SpecJob co;
        co.in_field = FS_U;
        co.nin = D;
        co.nout = D;
        for (int a = 0; a < D; ++a) co.op[a] = OpSpec{AO_COLLOC, (int8_t)a, RT_NONE, (int8_t)a};
        co.spec_in = sp1;
        co.spec_out = sp1;
        co.epi = EPI_STORE;
        co.out_field = FS_TMP;
        co.gate = GATE_RECU;
        co.name = "colloc";
        issue_job(co, -1);
        if (!tune_mode_ && !dry_)
            for (int a = 0; a < D; ++a) launch_sample(st(), d_sims_, d_t_, count(), max_pts_, 1, a);
    }
    if (!tick_in_sample) timed("tick", 0, [&] { launch_tick(st(), d_t_); });
}

bool Engine::host_gate(const SimHost& h, int gate, int comp) const {
    const SimDev& S = h.dev;
    if (t_ >= h.nt) return false;
    switch (gate) {
        case GATE_PSRC: return S.has_p && !S.psrc_q && t_ < S.psrc.len;
        case GATE_USRC: return comp < h.dim && S.has_u[comp] && t_ < S.usrc[comp].len;
        case GATE_P0: return S.has_p0 != 0;
        case GATE_ABS: return comp == 0 ? S.absorb >= 2 : S.absorb == 3;
        case GATE_RECU: return S.sensor.kind != 0 && (S.sensor.record_u_series || S.sensor.record_u_agg);
        default: return gate >= GATE_DIR ? gate - GATE_DIR < S.sensor.ndir : true;
    }
}

// Compulsory HBM bytes per grid point of a C2R epilogue (field reads and writes; scalars and
// per-axis vectors cost nothing).
double Engine::epi_bytes(const SimHost& h, int epi, int ncomp) const {
    const SimDev& S = h.dev;
    auto m = [](const FieldOrScalar& f) { return f.ptr ? 4.0 : 0.0; };
    const int D = h.dim;
    double eos = 4 + m(S.c2) + (S.absorb == 1 ? m(S.tau) : 0) + (S.nonlinear ? m(S.bona) : 0);
    switch (epi) {
        case EPI_STORE: return 4.0 * ncomp;
        case EPI_VEL: { double b = 0; for (int a = 0; a < ncomp; ++a) b += 8 + m(S.dtor[a]); return b; }
        case EPI_VEL_INIT: { double b = 0; for (int a = 0; a < ncomp; ++a) b += 4 + m(S.dtor[a]); return b; }
        case EPI_ADD_U: return 8.0 * ncomp;
        case EPI_DEN:
        case EPI_DEN_SRC:
            return 8.0 * D + 4 + m(S.rho0) + (S.absorb >= 1 ? 4 : 0) + (S.eos_pointwise ? eos : 0) +
                   (epi == EPI_DEN_SRC && S.psrc_q && t_ < S.psrc.len ? 4 : 0);
        case EPI_ADD_RHO: return 8.0 * D + 4 + (S.eos_pointwise ? eos + (S.absorb == 1 ? 4 : 0) : 0);
        case EPI_EOS_ABS:
            return 8 + m(S.c2) + m(S.tau) + (S.absorb == 3 ? m(S.eta) : 0) + (S.nonlinear ? m(S.bona) + m(S.rho0) : 0);
        default: return 0;
    }
}

// Number of fields the C2R epilogue `epi` stages per row (an upper bound of the device-side plan:
// velocity u / dt/rho_sg; density rho_a, rho0, and the pointwise EoS inputs; power-law EoS inputs).
int Engine::aux_slots(const SimHost& h, int epi) const {
    const SimDev& S = h.dev;
    auto m = [](const FieldOrScalar& f) { return f.ptr ? 1 : 0; };
    switch (epi) {
        case EPI_VEL: return 2;
        case EPI_VEL_INIT: return 1;
        case EPI_ADD_U: return 1;
        case EPI_DEN:
        case EPI_DEN_SRC:
        case EPI_ADD_RHO:
            return h.dim + 1 + (S.eos_pointwise ? m(S.c2) + (S.absorb == 1 ? m(S.tau) + 1 : 0) + (S.nonlinear ? m(S.bona) : 0) : 0);
        case EPI_EOS_ABS:
            return 1 + m(S.c2) + m(S.tau) + (S.absorb == 3 ? m(S.eta) : 0) + (S.nonlinear ? m(S.bona) + m(S.rho0) : 0);
        default: return 0;
    }
}

std::vector<Engine::KernelTiming> Engine::profile_step(int reps) {
    std::vector<KernelTiming> acc;
    int tmax = 0;
    for (auto& h : sims_) tmax = std::max(tmax, h.nt);
    int done = 0;
    for (int r = 0; r < reps && t_ < tmax; ++r) {
        if (t_ == 0) { step(1); continue; }
        std::vector<ProfRec> recs;
        prof_ = &recs;
        try {
            issue_step(false);
        } catch (...) {
            prof_ = nullptr;
            throw;
        }
        prof_ = nullptr;
        ++t_;
        check(cudaStreamSynchronize(st()), "profile sync");
        if (acc.empty()) acc.resize(recs.size());
        for (size_t i = 0; i < recs.size() && i < acc.size(); ++i) {
            float ms = 0;
            cudaEventElapsedTime(&ms, recs[i].a, recs[i].b);
            acc[i].name = recs[i].name;
            acc[i].bytes = recs[i].bytes;
            acc[i].ms += ms;
            cudaEventDestroy(recs[i].a);
            cudaEventDestroy(recs[i].b);
        }
        ++done;
    }
    for (auto& k : acc) k.ms /= std::max(done, 1);
    return acc;
}

// true while some simulation's precorrected pressure source still injects at step t_
bool Engine::psrc_live() const {
    for (const auto& h : sims_)
        if (h.dev.psrc_q && h.dev.has_p && t_ < h.dev.psrc.len && t_ < h.nt) return true;
    return false;
}

int Engine::capture_graph() {
    const int var = psrc_live() ? 1 : 0;
    if (graph_exec_[var] && graph_stream_[var] == st()) return var;
    if (graph_exec_[var]) { cudaGraphExecDestroy(graph_exec_[var]); graph_exec_[var] = nullptr; }
    if (graph_[var]) { cudaGraphDestroy(graph_[var]); graph_[var] = nullptr; }
    // a dry pass first: it creates every tile map this step variant needs (device allocations are
    // not allowed inside the capture) and launches nothing. The axisymmetric step launches its own
    // kernels directly and has one job structure, whose maps its first (uncaptured) step created.
    if (!as_mode_) {
        dry_ = true;
        try {
            issue_step(false);
        } catch (...) {
            dry_ = false;
            throw;
        }
        dry_ = false;
    }
    check(cudaStreamBeginCapture(st(), cudaStreamCaptureModeThreadLocal), "begin capture");
    try {
        issue_step(false);
    } catch (...) {
        cudaGraph_t g;
        cudaStreamEndCapture(st(), &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    check(cudaStreamEndCapture(st(), &graph_[var]), "end capture");
    check(cudaGraphInstantiate(&graph_exec_[var], graph_[var], 0), "graph instantiate");
    graph_stream_[var] = st();
    return var;
}

// ------------------------------------------------------------------------------------------
// setup of one simulation
// ------------------------------------------------------------------------------------------
void Engine::smooth_field(int s, float* field) {
    // smooth(..., restore_max): Re F^-1(W F(f)) * max|f| / max|out| (Filter/Filters.swift:273-347).
    // The window is applied as its Hermitian part (W(k) + W(-k))/2, which gives exactly the real
    // part the reference takes.
    SimHost& h = sims_[s];
    check(cudaMemcpyAsync(h.dev.tmp[0], field, h.N * sizeof(float), cudaMemcpyDeviceToDevice, st()), "copy");
    check(cudaMemsetAsync(d_red_, 0, 2 * sizeof(unsigned int), st()), "memset");
    launch_absmax(st(), h.dev.tmp[0], h.N, d_red_);
    SpecJob sj;
    sj.in_field = FS_TMP;
    sj.nin = 1;
    sj.nout = 1;
    sj.op[0] = OpSpec{AO_NONE, 0, RT_WINDOW, 0};
    sj.epi = EPI_STORE;
    sj.out_field = FS_TMP;
    sj.name = "smooth";
    issue_job(sj, s);
    launch_absmax(st(), h.dev.tmp[0], h.N, d_red_ + 1);
    launch_scale(st(), h.dev.tmp[0], h.N, d_red_, d_red_ + 1);
    check(cudaMemcpyAsync(field, h.dev.tmp[0], h.N * sizeof(float), cudaMemcpyDeviceToDevice, st()), "copy");
}

void Engine::setup_sim(int s, const kw_sim_desc& d) {
    SimHost& h = sims_[s];
    h.d = d;
    if (d.abi_version != KW_ABI_VERSION) throw err(KW_ERR_INVALID, "descriptor abi_version mismatch");
    if (d.dim < 1 || d.dim > 3) throw err(KW_ERR_INVALID, "kspaceFirstOrder: dim " + std::to_string(d.dim) + " not yet implemented");
    h.dim = d.dim;
    const int nref[3] = {d.nx, d.ny, d.nz};
    const double dref[3] = {d.dx, d.dy, d.dz};
    for (int a = 0; a < h.dim; ++a) {
        if (nref[a] < 1) throw err(KW_ERR_INVALID, "grid size must be positive");
        if (!(dref[a] > 0)) throw err(KW_ERR_INVALID, "grid spacing must be positive");
        if (nref[a] > 4096) throw err(KW_ERR_UNSUPPORTED, "axis length above 4096");
        h.n_ref[a] = nref[a];
        h.d_ref[a] = dref[a];
    }
    if (d.nt <= 0) throw err(KW_ERR_INVALID, "call grid.makeTime(...) before running the solver");
    if (!(d.dt > 0)) throw err(KW_ERR_INVALID, "dt must be positive");
    if (!d.p0 && !d.p_mask && !d.u_mask)
        throw err(KW_ERR_INVALID, std::to_string(h.dim) + "D solver requires source.p0 or a time-varying p/u source");
    h.nt = d.nt;
    if (h.dim == 1) { h.A = 1; h.B = 1; h.C = d.nx; }
    else if (h.dim == 2) { h.A = 1; h.B = d.nx; h.C = d.ny; }
    else { h.A = d.nx; h.B = d.ny; h.C = d.nz; }
    h.N = (long long)h.A * h.B * h.C;
    if (h.N > (1LL << 31) - 1) throw err(KW_ERR_UNSUPPORTED, "grids above 2^31 points are not supported");
    h.Ch = h.C / 2 + 1;
    h.Cp = (h.Ch + 3) & ~3;   // a multiple of 4 (16-byte rows of the float radial tables)
    h.Ns = (long long)h.A * h.B * h.Cp;
    const long long N = h.N;
    auto grid_sized = [&](const kw_array& a) { return a.data && (a.len == 1 || (long long)a.len == N); };
    if (!grid_sized(d.sound_speed)) throw err(KW_ERR_INVALID, "soundSpeed must be scalar or grid-shaped");
    if (!grid_sized(d.density)) throw err(KW_ERR_INVALID, "density must be scalar or grid-shaped");
    if (d.pml_size < 0) throw err(KW_ERR_INVALID, "pmlSize must be non-negative");
    for (int a = 0; a < h.dim; ++a)
        if (d.pml_size > h.n_ref[a]) throw err(KW_ERR_INVALID, "pmlSize larger than the grid");
    if (d.alpha_coeff.data && !grid_sized(d.alpha_coeff)) throw err(KW_ERR_INVALID, "alphaCoeff must be scalar or grid-shaped");
    if (d.b_on_a.data && !grid_sized(d.b_on_a)) throw err(KW_ERR_INVALID, "bOnA must be scalar or grid-shaped");

    SimDev& v = h.dev;
    std::memset(&v, 0, sizeof(v));
    v.dim = h.dim; v.A = h.A; v.B = h.B; v.C = h.C; v.Ch = h.Ch; v.Cp = h.Cp;
    v.N = h.N; v.Ns = h.Ns; v.nt = h.nt;
    v.inv_n = (float)(1.0 / (double)N);
    for (int L = 0; L < 3; ++L) v.axis_of_layout[L] = L + h.dim - 3;

    trace_phase("validate");
    // FFT plans
    const bool odd = (h.C & 1) != 0;
    build_plan(v.plan_row, odd ? h.C : h.C / 2);
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
    max_A_ = std::max(max_A_, h.A);
    max_B_ = std::max(max_B_, h.B);
    h.M = odd ? h.C : h.C / 2;
    max_M_ = std::max(max_M_, h.M);

    trace_phase("plans");
    // device fields
    const size_t fb = (size_t)N * sizeof(float);
    const int nspec = h.dim + 1;
    for (int i = 0; i < nspec; ++i) v.spec[i] = (float2*)dalloc((size_t)h.Ns * sizeof(float2));
    v.p = (float*)dalloc(fb);
    v.rho_sum = (float*)dalloc(fb);
    for (int a = 0; a < h.dim; ++a) {
        v.u[a] = (float*)dalloc(fb);
        v.rho[a] = (float*)dalloc(fb);
    }
    v.tmp[0] = (float*)dalloc(fb);
    v.nonfinite = d_flag_;
    v.wait_cycles = wait_cycles_;
    v.test_stall = test_stall_;

    trace_phase("alloc fields");
    // ---- medium; smoothing on the device (KSFO:367-373) ----
    const bool c0map = d.sound_speed.len > 1, rho0map = d.density.len > 1;
    // FP64 host copies only of smoothed maps (their values come back from the device); an
    // unsmoothed map is read from the caller's buffer where the host needs single values
    const bool c0_host = c0map && d.smooth_c0;
    std::vector<double> c0(c0_host ? N : 1), rho0(rho0map && d.smooth_rho0 ? N : 1);
    c0[0] = d.sound_speed.data[0];
    auto smooth_to_host = [&](const float* src, std::vector<double>& dst) {
        float* f = (float*)dalloc(fb);
        upload_host(f, src, fb);
        // the smoothing job needs the device descriptor (plans, buffers, window)
        check(cudaMemcpyAsync(d_sims_ + s, &v, sizeof(SimDev), cudaMemcpyHostToDevice, st()), "upload sim");
        smooth_field(s, f);
        std::vector<float> host(N);
        check(cudaMemcpyAsync(host.data(), f, fb, cudaMemcpyDeviceToHost, st()), "download");
        check(cudaStreamSynchronize(st()), "sync");
        parallel_for(N, [&](long long i) { dst[i] = host[i]; });
        return f;
    };
    const bool need_window = (d.smooth_c0 && c0map) || (d.smooth_rho0 && rho0map) || (d.p0 && d.smooth_p0);
    if (need_window) {
        // FFT-order smoothing window of the reference (Filters.swift:218-321), Hermitian part,
        // over the half spectrum. 2D fills out[i][j] = win[(i+sx)%nx][(j+sy)%ny]; 1D/3D fill
        // out[(i+sx)%n] = win[i]; both are reproduced.
        std::vector<int> enl(h.dim);
        int Lw = 1;
        for (int a = 0; a < h.dim; ++a) { enl[a] = h.n_ref[a] % 2 ? h.n_ref[a] : h.n_ref[a] + 1; Lw = std::max(Lw, enl[a]); }
        std::vector<double> winLin(Lw, 1.0);
        if (Lw > 1)
            for (int i = 0; i < Lw; ++i) {
                const double x = 2.0 * M_PI * (double)i / (double)(Lw - 1);
                winLin[i] = 0.42 - 0.5 * std::cos(x) + 0.08 * std::cos(2.0 * x);
            }
        const double radius = (double)(Lw - 1) / 2.0;
        std::vector<std::vector<double>> pos(h.dim);   // window-axis coordinate of FFT-order index m
        for (int a = 0; a < h.dim; ++a) {
            const int n = h.n_ref[a], cnt = enl[a];
            const int sx = (n + 1) / 2;
            pos[a].resize(n);
            for (int m = 0; m < n; ++m) {
                const int wi = h.dim == 2 ? (m + sx) % n : ((m - sx) % n + n) % n;
                pos[a][m] = cnt <= 1 ? 0.0 : -radius + 2.0 * radius * (double)wi / (double)(cnt - 1);
            }
        }
        auto interp = [&](double r) {
            const double p = std::min(r, radius) + radius;
            const int i0 = std::min((int)std::floor(p), (int)winLin.size() - 2);
            if (winLin.size() < 2) return 1.0;
            const double fr = p - (double)i0;
            return std::fabs(winLin[i0] * (1.0 - fr) + winLin[i0 + 1] * fr);
        };
        auto W = [&](const int* m) {
            double r2 = 0;
            for (int a = 0; a < h.dim; ++a) r2 += pos[a][m[a]] * pos[a][m[a]];
            return interp(std::sqrt(r2));
        };
        std::vector<float> tab((size_t)h.Ns, 0.f);
        parallel_for((long long)h.A * h.B * h.Ch, [&](long long q) {
            const int kc = (int)(q % h.Ch);
            const long long r = q / h.Ch;
            const int ib = (int)(r % h.B), ia = (int)(r / h.B);
            int lay[3] = {ia, ib, kc}, ln[3] = {h.A, h.B, h.C};
            int m[3], mm[3];
            for (int a = 0; a < h.dim; ++a) {
                const int L = a + 3 - h.dim;
                m[a] = lay[L];
                mm[a] = (ln[L] - lay[L]) % ln[L];
            }
            tab[((size_t)ia * h.B + ib) * h.Cp + kc] = (float)(0.5 * (W(m) + W(mm)));
        });
        v.radial[RT_WINDOW] = upload(tab);
        build_tensor_maps(h, v);   // the smoothing jobs below run the TMA-fed column pass
    }
    // the (smoothed) maps stay on the device: the medium-derived fields are computed there in FP64
    // (kw_setup.cu); the host keeps c0 for c_ref and the source scales
    float* d_c0 = nullptr;
    float* d_rho0 = nullptr;
    if (c0_host) d_c0 = smooth_to_host(d.sound_speed.data, c0);
    else if (c0map) d_c0 = upload_floats(d.sound_speed.data, N);
    if (d.smooth_rho0 && rho0map) d_rho0 = smooth_to_host(d.density.data, rho0);
    else if (rho0map) d_rho0 = upload_floats(d.density.data, N);
    else rho0[0] = d.density.data[0];
    if (d.p0) {
        float* f = (float*)dalloc(fb);
        upload_host(f, d.p0, fb);
        if (d.smooth_p0) {
            check(cudaMemcpyAsync(d_sims_ + s, &v, sizeof(SimDev), cudaMemcpyHostToDevice, st()), "upload sim");
            smooth_field(s, f);
        }
        h.p0s = f;
        v.has_p0 = 1;
    }
    auto c0_at = [&](long long i) -> double { return c0_host ? c0[i] : (c0map ? (double)d.sound_speed.data[i] : c0[0]); };

    trace_phase("medium upload");
    // referenceSoundSpeed (KSFO:786-788), or the caller's fixed value
    double cref = c0[0];
    if (c0map && !c0_host) {   // the largest value of the map, on the device (exact: a max)
        check(cudaMemsetAsync(d_red_ + 2, 0, sizeof(unsigned int), st()), "memset");
        launch_setup_max(st(), d_c0, N, d_red_ + 2);
        unsigned int bits = 0;
        check(cudaMemcpyAsync(&bits, d_red_ + 2, sizeof bits, cudaMemcpyDeviceToHost, st()), "c_ref");
        check(cudaStreamSynchronize(st()), "c_ref");
        cref = std::max(cref, (double)setup_max_decode(bits));
    } else if (c0map) {
        const long long nchunk = 64, per = (N + nchunk - 1) / nchunk;
        std::vector<double> part(nchunk, c0[0]);
        parallel_for(nchunk, [&](long long ch) {
            double m = c0[0];
            for (long long i = ch * per; i < std::min(N, (ch + 1) * per); ++i) m = std::max(m, c0[i]);
            part[ch] = m;
        });
        for (double x : part) cref = std::max(cref, x);
    }
    if (!std::isnan(d.c_ref)) cref = d.c_ref;
    h.cref = cref;
    const double dt = d.dt;

    trace_phase("c_ref");
    // ---- per-axis operators, PML (KSFO:376-397, 764-769) ----
    std::vector<std::vector<double>> kv(h.dim);
    for (int a = 0; a < h.dim; ++a) {
        const int n = h.n_ref[a];
        const double dd = h.d_ref[a];
        kv[a] = wavenumbers(n, dd);
        std::vector<float2> dp(n), dn(n), co(n);
        for (int i = 0; i < n; ++i) {
            const double k = kv[a][i], th = k * (dd / 2.0);
            const bool nyq = (n % 2 == 0) && i == n / 2;   // self-conjugate bin: Hermitian part
            dp[i] = make_float2((float)(-k * std::sin(th)), nyq ? 0.f : (float)(k * std::cos(th)));
            dn[i] = make_float2((float)(k * std::sin(th)), nyq ? 0.f : (float)(k * std::cos(th)));
            co[i] = make_float2((float)std::cos(th), nyq ? 0.f : (float)(-std::sin(th)));
        }
        AxisDev& ax = v.ax[a];
        ax.n = n;
        ax.dpos = upload(dp);
        ax.dneg = upload(dn);
        ax.colloc = upload(co);
        ax.pml = upload(to_f32(pml_profile(n, dd, dt, cref, d.pml_size, d.pml_alpha, false)));
        ax.pml_sg = upload(to_f32(pml_profile(n, dd, dt, cref, d.pml_size, d.pml_alpha, true)));
        ax.inv_d = (float)(1.0 / dd);
    }

    trace_phase("axis tables");
    // ---- medium-derived quantities ----
    // maps computed on the device in FP64 (kw_setup.cu), scalars here
    if (c0map) {
        float* c2 = (float*)dalloc(fb);
        launch_setup_c2(st(), d_c0, c2, N);
        v.c2 = FieldOrScalar{c2, 0.f};
    } else {
        v.c2 = FieldOrScalar{nullptr, (float)(c0[0] * c0[0])};
    }
    v.dt = (float)dt;
    v.rho0 = rho0map ? FieldOrScalar{d_rho0, 0.f} : FieldOrScalar{nullptr, (float)rho0[0]};
    for (int a = 0; a < h.dim; ++a) {
        // staggerDensity (KSFO:799-806): mean of neighbours, last index replicated
        const int L = a + 3 - h.dim;
        const long long stride = L == 2 ? 1 : (L == 1 ? h.C : (long long)h.B * h.C);
        const int n = h.n_ref[a];
        if (rho0map) {
            float* q = (float*)dalloc(fb);
            launch_setup_dtor(st(), d_rho0, q, N, stride, n, dt);
            v.dtor[a] = FieldOrScalar{q, 0.f};
        } else {
            v.dtor[a] = FieldOrScalar{nullptr, (float)(dt / rho0[0])};
        }
    }
    check(cudaGetLastError(), "setup kernels");

    // absorption (KSFO:851-882)
    v.absorb = 0;
    double y = 1.5;
    if (d.alpha_coeff.data && d.alpha_mode != KW_ABSORPTION_NONE) {
        y = std::isnan(d.alpha_power) ? 1.5 : d.alpha_power;
        if (d.alpha_mode == KW_ABSORPTION_STOKES) y = 2.0;
        const bool amap = d.alpha_coeff.len > 1;
        const double np1 = db2neper(1.0, y);
        auto anp = [&](long long i) { return (double)d.alpha_coeff.data[amap ? i : 0] * np1; };
        const bool stokes = d.alpha_mode == KW_ABSORPTION_STOKES || std::fabs(y - 2.0) < 1e-10;
        v.absorb = stokes ? 1 : (d.alpha_mode == KW_ABSORPTION_NO_DISPERSION ? 2 : 3);
        const double tn = std::tan(M_PI * y / 2.0);
        if (amap || c0map) {   // on the device in FP64 (kw_setup.cu)
            const float* d_alpha = amap ? upload_floats(d.alpha_coeff.data, N) : nullptr;
            float* tau = (float*)dalloc(fb);
            float* eta = v.absorb == 3 ? (float*)dalloc(fb) : nullptr;
            launch_setup_absorb(st(), c0map ? d_c0 : nullptr, c0[0], d_alpha, (double)d.alpha_coeff.data[0], np1, y,
                                stokes ? 1 : 0, tn, tau, eta, N);
            check(cudaGetLastError(), "setup absorption");
            v.tau = FieldOrScalar{tau, 0.f};
            if (eta) v.eta = FieldOrScalar{eta, 0.f};
        } else if (stokes) {
            v.tau = FieldOrScalar{nullptr, (float)(-2.0 * anp(0) * c0[0])};
        } else {
            v.tau = FieldOrScalar{nullptr, (float)(-2.0 * anp(0) * std::pow(c0[0], y - 1.0))};
            if (v.absorb == 3) v.eta = FieldOrScalar{nullptr, (float)(2.0 * anp(0) * std::pow(c0[0], y) * tn)};
        }
        v.div_term = (float*)dalloc(fb);
    }
    v.eos_pointwise = v.absorb < 2 ? 1 : 0;
    // nonlinearity (KSFO:902-907)
    v.nonlinear = 0;
    if (d.b_on_a.data) {
        const bool bmap = d.b_on_a.len > 1;
        double mx = 0;
        for (size_t i = 0; i < d.b_on_a.len; ++i) mx = std::max(mx, (double)std::fabs(d.b_on_a.data[i]));
        if (mx != 0.0) {
            v.nonlinear = 1;
            v.bona = bmap ? FieldOrScalar{upload_floats(d.b_on_a.data, N), 0.f} : FieldOrScalar{nullptr, d.b_on_a.data[0]};
        }
    }

    trace_phase("medium fields");
    // ---- sources (KSFO:404-423, 129-201) ----
    const double nd = (double)h.dim;
    bool need_skappa = false;
    if (d.p_mask && d.p.data) {
        std::vector<int> idx = flat_nonzero(d.p_mask, N);
        if (!idx.empty()) {
            if (d.p.rows != 1 && d.p.rows != (int)idx.size())
                throw err(KW_ERR_INVALID, "source.p rows must be 1 or the number of source points");
            if (d.p.len < 0) throw err(KW_ERR_INVALID, "source.p length must be non-negative");
            SourceDev& sd = v.psrc;
            sd.nsrc = (int)idx.size();
            sd.rows = d.p.rows;
            sd.len = d.p.len;
            sd.mode = d.p_mode;
            sd.idx = upload(idx);
            sd.signal = upload(std::vector<float>(d.p.data, d.p.data + (size_t)d.p.rows * std::max(d.p.len, 0)));
            if (d.p_mode == KW_SOURCE_DIRICHLET) {
                std::vector<float> sc(idx.size());
                for (size_t q = 0; q < idx.size(); ++q) { const double c = c0_at(idx[q]); sc[q] = (float)(1.0 / (nd * c * c)); }
                sd.scale[0] = upload(sc);
            } else if (d.p_mode == KW_SOURCE_ADDITIVE_NO_CORRECTION) {
                for (int a = 0; a < h.dim; ++a) {
                    std::vector<float> sc(idx.size());
                    for (size_t q = 0; q < idx.size(); ++q) sc[q] = (float)(2.0 * dt / (nd * c0_at(idx[q]) * h.d_ref[a]));
                    sd.scale[a] = upload(sc);
                }
            } else {
                std::vector<float> sc(idx.size());
                for (size_t q = 0; q < idx.size(); ++q) sc[q] = (float)(2.0 * dt / (nd * c0_at(idx[q])));
                sd.scale[0] = upload(sc);
                v.src_buf[0] = (float*)dalloc(fb);
                need_skappa = true;
                // one signal row: the corrected source is signal[t] times a fixed field
                h.psrc_precorrect = precorrect_ok_ && d.p.rows == 1 && d.p.len > 0;
                if (!h.psrc_precorrect) any_p_add_ = true;
            }
            if (d.p_mode != KW_SOURCE_ADDITIVE) any_p_direct_ = true;
            v.has_p = sd.len > 0;
            max_psrc_ = std::max(max_psrc_, sd.nsrc);
        }
    }
    if (d.u_mask) {
        std::vector<int> idx = flat_nonzero(d.u_mask, N);
        const kw_signal* sig[3] = {&d.ux, &d.uy, &d.uz};
        if (!idx.empty()) {
            int* didx = upload(idx);
            for (int a = 0; a < h.dim; ++a) {
                if (!sig[a]->data) continue;
                if (sig[a]->rows != 1 && sig[a]->rows != (int)idx.size())
                    throw err(KW_ERR_INVALID, "source velocity rows must be 1 or the number of source points");
                SourceDev& sd = v.usrc[a];
                sd.nsrc = (int)idx.size();
                sd.rows = sig[a]->rows;
                sd.len = std::max(sig[a]->len, 0);
                sd.mode = d.u_mode;
                sd.idx = didx;
                sd.signal = upload(std::vector<float>(sig[a]->data, sig[a]->data + (size_t)sd.rows * sd.len));
                std::vector<float> sc(idx.size());
                for (size_t q = 0; q < idx.size(); ++q)
                    sc[q] = d.u_mode == KW_SOURCE_DIRICHLET ? 1.f : (float)(2.0 * c0_at(idx[q]) * dt / h.d_ref[a]);
                sd.scale[0] = upload(sc);
                if (d.u_mode == KW_SOURCE_ADDITIVE) {
                    v.src_buf[a] = (float*)dalloc(fb);
                    need_skappa = true;
                    any_u_add_ = true;
                } else {
                    any_u_direct_ = true;
                }
                v.has_u[a] = sd.len > 0;
                max_usrc_ = std::max(max_usrc_, sd.nsrc);
            }
        }
    }

    trace_phase("sources");
    // ---- radial tables over the half spectrum (FP64 -> FP32) ----
    {
        std::vector<double> kA(h.A, 0.0), kB(h.B, 0.0), kC(h.C, 0.0);
        for (int a = 0; a < h.dim; ++a) {
            const int L = a + 3 - h.dim;
            std::vector<double>& dst = L == 0 ? kA : (L == 1 ? kB : kC);
            dst = kv[a];
        }
        // computed on the device in FP64 from the wavenumber vectors (kw_setup.cu); the padding
        // bins keep dalloc's zeros
        const size_t tb = (size_t)h.Ns * sizeof(float);
        float* kap = (float*)dalloc(tb);
        float* skap = need_skappa ? (float*)dalloc(tb) : nullptr;
        float* nu1 = v.absorb >= 2 ? (float*)dalloc(tb) : nullptr;
        float* nu2 = v.absorb == 3 ? (float*)dalloc(tb) : nullptr;
        const double* dkA = upload(kA);
        const double* dkB = upload(kB);
        const double* dkC = upload(kC);
        launch_setup_radial(st(), dkA, dkB, dkC, h.A, h.B, h.Ch, h.Cp, cref * dt / 2.0, y, kap, skap, nu1, nu2);
        check(cudaGetLastError(), "setup radial tables");
        v.radial[RT_KAPPA] = kap;
        v.radial[RT_SKAPPA] = skap;
        v.radial[RT_NU1] = nu1;
        v.radial[RT_NU2] = nu2;
    }

    trace_phase("radial tables");
    // ---- sensor (REC:8-97) ----
    const unsigned rec = d.record;
    h.record_p = (rec & (KW_RECORD_P | KW_RECORD_P_MAX | KW_RECORD_P_MIN | KW_RECORD_P_RMS | KW_RECORD_I_AVG)) != 0;
    h.record_u = (rec & (KW_RECORD_UX | KW_RECORD_UY | KW_RECORD_UZ | KW_RECORD_U_MAX | KW_RECORD_U_RMS | KW_RECORD_I_AVG)) != 0;
    h.record_ufinal = (rec & KW_RECORD_U_FINAL) != 0;
    SensorDev& sn = v.sensor;
    if (d.sensor_mask && (d.sensor_kind == KW_SENSOR_BINARY || d.sensor_kind == KW_SENSOR_CARTESIAN)) {
        if (d.sensor_kind == KW_SENSOR_BINARY) {
            std::vector<int> idx = flat_nonzero(d.sensor_mask, N);
            sn.kind = 1;
            sn.npts = (int)idx.size();
            sn.ncorners = 1;
            sn.idx = upload(idx);
        } else {
            if (d.sensor_points < 0) throw err(KW_ERR_INVALID, "sensor_points must be non-negative");
            const int np = d.sensor_points, nc = 1 << h.dim;
            std::vector<int> idx((size_t)np * nc);
            std::vector<float> w((size_t)np * nc);
            for (int p = 0; p < np; ++p) {
                int i0[3];
                double fr[3];
                for (int a = 0; a < h.dim; ++a) {
                    const double g = (double)d.sensor_mask[(size_t)a * np + p] / h.d_ref[a] + (double)(h.n_ref[a] / 2);
                    if (!(g >= 0 && g <= (double)(h.n_ref[a] - 1)))
                        throw err(KW_ERR_INVALID, "Cartesian sensor point outside grid bounds (axis " + std::to_string(a) + ")");
                    const double f = std::floor(g);
                    i0[a] = (int)f;
                    fr[a] = g - f;
                }
                for (int c = 0; c < nc; ++c) {
                    long long flat = 0;
                    double ww = 1.0;
                    for (int a = 0; a < h.dim; ++a) {
                        const int bit = (c >> a) & 1;
                        const int ai = std::min(i0[a] + bit, h.n_ref[a] - 1);
                        ww *= bit == 1 ? fr[a] : (1.0 - fr[a]);
                        flat = flat * h.n_ref[a] + ai;
                    }
                    idx[(size_t)p * nc + c] = (int)flat;
                    w[(size_t)p * nc + c] = (float)ww;
                }
            }
            sn.kind = 2;
            sn.npts = np;
            sn.ncorners = nc;
            sn.idx = upload(idx);
            sn.w = upload(w);
        }
        h.npts = sn.npts;
        h.p_series = h.record_p && (rec & (KW_RECORD_P | KW_RECORD_I_AVG));
        h.p_agg = h.record_p && (rec & (KW_RECORD_P_MAX | KW_RECORD_P_MIN | KW_RECORD_P_RMS));
        h.u_series = h.record_u && (rec & (KW_RECORD_UX | KW_RECORD_UY | KW_RECORD_UZ | KW_RECORD_I_AVG));
        h.u_agg = h.record_u && (rec & (KW_RECORD_U_MAX | KW_RECORD_U_RMS));
        sn.record_p_series = h.p_series;
        sn.record_p_agg = h.p_agg;
        sn.record_u_series = h.u_series;
        sn.record_u_agg = h.u_agg;
        const size_t np = (size_t)std::max(sn.npts, 1);
        if (h.p_series) sn.p_series = (float*)dalloc((size_t)h.nt * np * sizeof(float));
        if (h.p_agg) {
            sn.p_max = (float*)dalloc(np * 4); sn.p_min = (float*)dalloc(np * 4);
            sn.p_ss = (float*)dalloc(np * 4); sn.p_ssc = (float*)dalloc(np * 4);
        }
        if (h.record_u) {
            for (int a = 1; a < h.dim; ++a) v.tmp[a] = (float*)dalloc(fb);
            for (int a = 0; a < h.dim; ++a) {
                if (h.u_series) sn.u_series[a] = (float*)dalloc((size_t)h.nt * np * sizeof(float));
                if (h.u_agg) {
                    sn.u_max[a] = (float*)dalloc(np * 4);
                    sn.u_ss[a] = (float*)dalloc(np * 4);
                    sn.u_ssc[a] = (float*)dalloc(np * 4);
                }
            }
            any_recu_ = true;
        }
        if (h.record_p) any_recp_ = true;
        max_pts_ = std::max(max_pts_, sn.npts);

        // 2D directivity of binary sensors (Directivity.swift:41-79): per distinct angle th a
        // k-space weight W (pressure pattern: sinc of k along the element, size 10 max(dx, dy) by
        // default; gradient pattern: the normal component of k over |k|). The sampled value is
        // Re F^-1(W F(p)), i.e. the C2R of (W(k) + W(-k)) / 2 times the half spectrum.
        if (h.dim == 2 && d.sensor_kind == KW_SENSOR_BINARY && d.directivity_angle && sn.npts > 0 && h.record_p) {
            std::vector<int> gidx = flat_nonzero(d.sensor_mask, N);
            std::vector<double> rowAngle(gidx.size());
            for (size_t r = 0; r < gidx.size(); ++r) rowAngle[r] = (double)d.directivity_angle[gidx[r]];
            std::vector<double> uniq(rowAngle);
            std::sort(uniq.begin(), uniq.end());
            uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
            if ((int)uniq.size() > kMaxDirAngles)
                throw err(KW_ERR_UNSUPPORTED, "more than " + std::to_string(kMaxDirAngles) + " distinct directivity angles");
            const double elem = std::isnan(d.directivity_size) ? 10.0 * std::max(h.d_ref[0], h.d_ref[1]) : d.directivity_size;
            const std::vector<double>& kx = kv[0];   // reference axis 0: layout axis B
            const std::vector<double>& ky = kv[1];   // reference axis 1: layout axis C (rows)
            auto weight = [&](double th, double x, double y) {
                if (d.directivity_pattern == KW_DIRECTIVITY_PRESSURE) {
                    const double u = (std::cos(th) * y - std::sin(th) * x) * (elem / 2.0);
                    return u == 0.0 ? 1.0 : std::sin(M_PI * u) / (M_PI * u);
                }
                const double k = std::sqrt(x * x + y * y);
                return k == 0.0 ? 0.0 : (std::sin(th) * y + std::cos(th) * x) / k;
            };
            for (size_t j = 0; j < uniq.size(); ++j) {
                std::vector<float> tab((size_t)h.Ns, 0.f);
                for (int ib = 0; ib < h.B; ++ib)
                    for (int kc = 0; kc < h.Ch; ++kc) {
                        const int mb = (h.B - ib) % h.B, mc = (h.C - kc) % h.C;
                        const double w = 0.5 * (weight(uniq[j], kx[ib], ky[kc]) + weight(uniq[j], kx[mb], ky[mc]));
                        tab[(size_t)ib * h.Cp + kc] = (float)w;
                    }
                v.radial[RT_DIR0 + j] = upload(tab);
            }
            std::vector<int> slot(gidx.size());
            for (size_t r = 0; r < gidx.size(); ++r)
                slot[r] = (int)(std::lower_bound(uniq.begin(), uniq.end(), rowAngle[r]) - uniq.begin());
            sn.ndir = (int)uniq.size();
            sn.dir_slot = upload(slot);
            sn.dir_field = (float*)dalloc((size_t)sn.ndir * N * sizeof(float));
            max_dir_ = std::max(max_dir_, sn.ndir);
        }
    }
    if (v.absorb >= 2) any_abs_ = true;
    if (v.has_p0) any_p0_ = true;
    trace_phase("sensor");
    build_tensor_maps(h, v);
    check(cudaMemcpyAsync(d_sims_ + s, &v, sizeof(SimDev), cudaMemcpyHostToDevice, st()), "upload sim");
    trace_phase("tensor maps");
}

// The k-space corrected additive source of a single-row signal (SourceOp.apply .additive,
// KSpaceFirstOrder.swift:167-172) is linear in the signal value: for axis a at step t it is
// signal[t] Re F^-1(cos(c_ref dt k / 2) F(scale * mask)) / d_a with scale = 2 dt / (D c0). The
// field Q = Re F^-1(cos(.) F(scale * mask)) is computed here once, into the simulation's source
// buffer, and the density epilogue adds signal[t] Q / d_a to each rho_a: the per-step scatter and
// transform job of the source disappear.
void Engine::precorrect_psrc(int s) {
    SimHost& h = sims_[s];
    SimDev& v = h.dev;
    launch_scatter(st(), v.src_buf[0], v.psrc.idx, v.psrc.scale[0], v.psrc.nsrc);
    check(cudaGetLastError(), "source scatter");
    SpecJob q;
    q.in_field = FS_SRCBUF;
    q.nin = 1;
    q.nout = 1;
    q.op[0] = OpSpec{AO_NONE, 0, RT_SKAPPA, 0};
    q.epi = EPI_STORE;
    q.out_field = FS_SRCBUF;
    q.name = "psrc_q";
    issue_job(q, s);
    v.psrc_q = v.src_buf[0];
    check(cudaMemcpyAsync(d_sims_ + s, &v, sizeof(SimDev), cudaMemcpyHostToDevice, st()), "upload sim");
}

// KW_TRACE_SETUP=1: wall time since the previous mark, per phase of create, on stderr (the
// stream is synchronised first, so device work is counted where it was issued)
void Engine::trace_phase(const char* what) {
    if (!trace_) return;
    check(cudaStreamSynchronize(st()), "trace sync");
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "kw setup: %-16s %8.2f ms\n", what, std::chrono::duration<double, std::milli>(now - trace_last_).count());
    trace_last_ = now;
}

void Engine::create(const kw_sim_desc* descs, int n) {
    if (n <= 0) throw err(KW_ERR_INVALID, "no simulations");
    // kspaceFirstOrderAS: one simulation, its preconditions (KSpaceFirstOrderAS.swift:35-38,87-95),
    // p / pFinal recording only; a missing alphaPower means 2 there
    kw_sim_desc as_desc;
    bool as = false;
    for (int i = 0; i < n; ++i) as = as || descs[i].axisymmetric;
    if (as) {
        if (n != 1) throw err(KW_ERR_UNSUPPORTED, "axisymmetric simulations run one at a time");
        as_desc = descs[0];
        if (as_desc.dim != 2) throw err(KW_ERR_INVALID, "axisymmetric solver requires a 2D grid (x axial, y radial)");
        if (as_desc.nt <= 0) throw err(KW_ERR_INVALID, "call grid.makeTime(...) before running the solver");
        if (!as_desc.p0 && !as_desc.p_mask && !as_desc.u_mask)
            throw err(KW_ERR_INVALID, "axisymmetric solver requires source.p0 or a time-varying p/u source");
        if (as_desc.alpha_coeff.data && as_desc.alpha_mode != KW_ABSORPTION_NONE) {
            const double y = as_desc.alpha_mode == KW_ABSORPTION_STOKES ? 2.0
                             : (std::isnan(as_desc.alpha_power) ? 2.0 : as_desc.alpha_power);
            if (std::fabs(y - 2.0) >= 1e-10)
                throw err(KW_ERR_INVALID, "axisymmetric absorption requires the Stokes model (alphaPower = 2)");
            as_desc.alpha_mode = KW_ABSORPTION_STOKES;
        }
        as_desc.record &= (unsigned)(KW_RECORD_P | KW_RECORD_P_FINAL);
        as_desc.directivity_angle = nullptr;
        as_desc.axisymmetric = 0;
        descs = &as_desc;
        precorrect_ok_ = false;
    }
    check(cudaSetDevice(ctx_->device), "cudaSetDevice");
    sims_.resize(n);
    outs_.resize(n);
    dim_ = descs[0].dim;
    for (int i = 1; i < n; ++i)
        if (descs[i].dim != dim_) throw err(KW_ERR_INVALID, "all simulations of a batch must have the same dimensionality");
    d_sims_ = (SimDev*)dalloc(sizeof(SimDev) * n);
    d_t_ = (int*)dalloc(sizeof(int));
    d_flag_ = (int*)dalloc(2 * sizeof(int));   // [0] non-finite pressure, [1] device-side wait timeout
    d_tickc_ = (unsigned int*)dalloc(sizeof(unsigned int));   // CTAs of the step's last sample that have read t
    d_red_ = (unsigned int*)dalloc(4 * sizeof(unsigned int));
    const char* trace_env = std::getenv("KW_TRACE_SETUP");
    trace_ = trace_env && trace_env[0] == '1';
    trace_last_ = std::chrono::steady_clock::now();
    auto phase = [&](const char* what) { trace_phase(what); };
    for (int i = 0; i < n; ++i) setup_sim(i, descs[i]);
    phase("setup_sim");
    for (int i = 0; i < n; ++i)
        if (sims_[i].psrc_precorrect) precorrect_psrc(i);
    phase("precorrect");
    std::vector<const float*> p0s(n);
    for (int i = 0; i < n; ++i) p0s[i] = sims_[i].p0s;
    d_p0s_ = (const float**)dalloc(sizeof(float*) * n);
    check(cudaMemcpyAsync(d_p0s_, p0s.data(), sizeof(float*) * n, cudaMemcpyHostToDevice, st()), "upload");
    if (as) create_as_carrier();
    check(cudaStreamSynchronize(st()), "setup sync");
    reset();
    phase("reset");
    autotune();
    phase("autotune");
}

void Engine::reset() {
    for (auto& h : sims_) {
        const size_t fb = (size_t)h.N * sizeof(float);
        SimDev& v = h.dev;
        check(cudaMemsetAsync(v.p, 0, fb, st()), "reset");
        check(cudaMemsetAsync(v.rho_sum, 0, fb, st()), "reset");
        if (v.div_term) check(cudaMemsetAsync(v.div_term, 0, fb, st()), "reset");
        for (int a = 0; a < h.dim; ++a) {
            check(cudaMemsetAsync(v.u[a], 0, fb, st()), "reset");
            check(cudaMemsetAsync(v.rho[a], 0, fb, st()), "reset");
        }
        for (int a = 0; a < kMaxComp; ++a)
            if (v.src_buf[a] && v.src_buf[a] != v.psrc_q) check(cudaMemsetAsync(v.src_buf[a], 0, fb, st()), "reset");
    }
    check(cudaMemsetAsync(d_t_, 0, sizeof(int), st()), "reset");
    check(cudaMemsetAsync(d_tickc_, 0, sizeof(unsigned int), st()), "reset");
    check(cudaMemsetAsync(d_flag_, 0, 2 * sizeof(int), st()), "reset");
    t_ = 0;
    finalized_t_ = -1;
}

void Engine::step(int nsteps) {
    check(cudaGetLastError(), "pending error before step");
    int tmax = 0;
    for (auto& h : sims_) tmax = std::max(tmax, h.nt);
    nsteps = std::min(nsteps, tmax - t_);
    for (int k = 0; k < nsteps; ++k) {
        if (t_ == 0) {
            issue_step(true);
        } else {
            const int var = capture_graph();
            check(cudaGraphLaunch(graph_exec_[var], st()), "graph launch");
        }
        ++t_;
    }
    check(cudaGetLastError(), "launch");
}

// Test hooks, read once per engine from the environment (both off by default):
//   KW_TEST_STALL_COLUMN_PASS=1  the TMA-fed column pass withholds the copy of each CTA's first
//                                tile and its consumers wait at most ~20 us (40000 cycles) for it:
//                                the bounded wait runs out, the kernel records KE_TIMEOUT_FULL and
//                                returns, and the run reports KW_ERR_TIMEOUT;
//   KW_TEST_FAIL_ALLOC=n         the n-th device allocation fails as if the device were out of
//                                memory.
Engine::Engine(Context* ctx) : ctx_(ctx) {
    if (const char* w = std::getenv("KW_TEST_STALL_COLUMN_PASS"); w && w[0] == '1') {
        test_stall_ = 1;
        wait_cycles_ = 40000;
    }
    if (const char* f = std::getenv("KW_TEST_FAIL_ALLOC")) fail_alloc_ = std::max(0, std::atoi(f));
}

// kw_sim_run: every kFinitePoll steps the pressure of every simulation is checked for NaN / Inf
// on the device; the host reads that check's flag one poll later (it has long completed by then,
// so the stream never drains for it) and stops the run at the first poll that finds one, leaving
// synchronize() to report KW_ERR_NONFINITE.
void Engine::run(const kw_callbacks* cb) {
    reset();
    int tmax = 0;
    for (auto& h : sims_) tmax = std::max(tmax, h.nt);
    const int interval = cb && cb->monitor_interval > 0 ? cb->monitor_interval : 1;
    std::vector<float> host;
    if (!poll_host_) {
        check(cudaMallocHost(&poll_host_, sizeof(int)), "pinned flag");
        check(cudaEventCreateWithFlags(&poll_ev_, cudaEventDisableTiming), "event");
    }
    bool poll_pending = false;
    for (int t = 0; t < tmax; ++t) {
        if (t > 0 && t % kFinitePoll == 0) {
            if (poll_pending) {
                check(cudaEventSynchronize(poll_ev_), "poll");
                if (*poll_host_) break;
            }
            const Map& m = map_elems(-1);
            launch_check_finite(st(), d_sims_, d_t_, m.d, m.n);
            check(cudaMemcpyAsync(poll_host_, d_flag_, sizeof(int), cudaMemcpyDeviceToHost, st()), "poll copy");
            check(cudaEventRecord(poll_ev_, st()), "poll event");
            poll_pending = true;
        }
        step(1);
        if (cb && cb->monitor && t % interval == 0) {
            const SimHost& h = sims_[0];
            host.resize(h.N);
            check(cudaMemcpyAsync(host.data(), h.dev.p, h.N * sizeof(float), cudaMemcpyDeviceToHost, st()), "monitor copy");
            check(cudaStreamSynchronize(st()), "monitor sync");
            cb->monitor(t, host.data(), host.size(), cb->user);
        }
        if (cb && cb->progress) cb->progress(t, tmax, cb->user);
    }
}

int Engine::synchronize() {
    const Map& m = map_elems(-1);
    launch_check_finite(st(), d_sims_, d_t_, m.d, m.n);
    check(cudaStreamSynchronize(st()), "synchronize");
    check_kernel_error();
    int flag = 0;
    check(cudaMemcpy(&flag, d_flag_, sizeof(int), cudaMemcpyDeviceToHost), "flag");
    return flag ? KW_ERR_NONFINITE : KW_OK;
}

// A pass kernel whose bounded wait ran out leaves a code in d_flag_[1] (kw_async.cuh).
void Engine::check_kernel_error() {
    int code = 0;
    check(cudaMemcpy(&code, d_flag_ + 1, sizeof(int), cudaMemcpyDeviceToHost), "kernel error flag");
    if (code != 0)
        throw err(KW_ERR_TIMEOUT, "a device-side wait of a pass kernel timed out (code " + std::to_string(code) +
                                      "); the results of this run are invalid");
}

// ------------------------------------------------------------------------------------------
// outputs (REC:129-168)
// ------------------------------------------------------------------------------------------
static bool present(const SimHost& h, int f, int T) {
    const unsigned r = h.d.record;
    const bool smp = h.dev.sensor.kind != 0 && T > 0;
    const int a = (f - KW_FIELD_UX) % 3;
    switch (f) {
        case KW_FIELD_P: return smp && (r & KW_RECORD_P);
        case KW_FIELD_P_MAX: return smp && (r & KW_RECORD_P_MAX);
        case KW_FIELD_P_MIN: return smp && (r & KW_RECORD_P_MIN);
        case KW_FIELD_P_RMS: return smp && (r & KW_RECORD_P_RMS);
        case KW_FIELD_P_FINAL: return true;
        case KW_FIELD_UX: case KW_FIELD_UY: case KW_FIELD_UZ:
            return smp && a < h.dim && (r & (KW_RECORD_UX << a));
        case KW_FIELD_UX_MAX: case KW_FIELD_UY_MAX: case KW_FIELD_UZ_MAX:
            return smp && ((f - KW_FIELD_UX_MAX) < h.dim) && (r & KW_RECORD_U_MAX);
        case KW_FIELD_UX_RMS: case KW_FIELD_UY_RMS: case KW_FIELD_UZ_RMS:
            return smp && ((f - KW_FIELD_UX_RMS) < h.dim) && (r & KW_RECORD_U_RMS);
        case KW_FIELD_UX_FINAL: case KW_FIELD_UY_FINAL: case KW_FIELD_UZ_FINAL:
            return ((f - KW_FIELD_UX_FINAL) < h.dim) && (r & KW_RECORD_U_FINAL);
        case KW_FIELD_IX_AVG: case KW_FIELD_IY_AVG: case KW_FIELD_IZ_AVG:
            return smp && ((f - KW_FIELD_IX_AVG) < h.dim) && (r & KW_RECORD_I_AVG);
        default: return false;
    }
}

size_t Engine::output_size(int i, int f) const {
    const SimHost& h = sims_[i];
    const int T = std::min(t_, h.nt);
    if (!present(h, f, T)) return 0;
    switch (f) {
        case KW_FIELD_P: case KW_FIELD_UX: case KW_FIELD_UY: case KW_FIELD_UZ:
            return (size_t)h.npts * T;
        case KW_FIELD_P_FINAL: case KW_FIELD_UX_FINAL: case KW_FIELD_UY_FINAL: case KW_FIELD_UZ_FINAL:
            return (size_t)h.N;
        default:
            return (size_t)h.npts;
    }
}

const float* Engine::device_field(int i, int f, size_t* count) const {
    const SimHost& h = sims_[i];
    *count = (size_t)h.N;
    if (f == KW_FIELD_P_FINAL) return h.dev.p;
    if (f >= KW_FIELD_UX_FINAL && f <= KW_FIELD_UZ_FINAL && f - KW_FIELD_UX_FINAL < h.dim) return h.dev.u[f - KW_FIELD_UX_FINAL];
    *count = 0;
    return nullptr;
}

void Engine::get_output(int i, int f, float* dst, size_t count) {
    const SimHost& h = sims_[i];
    const int T = std::min(t_, h.nt);
    const size_t n = output_size(i, f);
    if (n == 0) throw err(KW_ERR_INVALID, "output field not recorded for this simulation");
    if (count != n) throw err(KW_ERR_INVALID, "output buffer size mismatch");
    const SensorDev& sn = h.dev.sensor;
    const size_t np = (size_t)h.npts;
    auto d2h = [&](const float* src, float* d, size_t cnt) { download_host(d, src, cnt * sizeof(float)); };
    auto series = [&](const float* dev) {   // [T][np] on the device -> [np][T] row-major
        std::vector<float> tmp((size_t)T * np);
        d2h(dev, tmp.data(), tmp.size());
        transpose_series(tmp.data(), dst, (size_t)T, np);
    };
    auto rms = [&](const float* ss) {
        std::vector<float> tmp(np);
        d2h(ss, tmp.data(), np);
        for (size_t q = 0; q < np; ++q) dst[q] = std::sqrt(tmp[q] / (float)T);
    };
    switch (f) {
        case KW_FIELD_P: series(sn.p_series); return;
        case KW_FIELD_P_MAX: d2h(sn.p_max, dst, np); break;
        case KW_FIELD_P_MIN: d2h(sn.p_min, dst, np); break;
        case KW_FIELD_P_RMS: rms(sn.p_ss); return;
        case KW_FIELD_P_FINAL: d2h(h.dev.p, dst, (size_t)h.N); break;
        case KW_FIELD_UX: case KW_FIELD_UY: case KW_FIELD_UZ: series(sn.u_series[f - KW_FIELD_UX]); return;
        case KW_FIELD_UX_MAX: case KW_FIELD_UY_MAX: case KW_FIELD_UZ_MAX: d2h(sn.u_max[f - KW_FIELD_UX_MAX], dst, np); break;
        case KW_FIELD_UX_RMS: case KW_FIELD_UY_RMS: case KW_FIELD_UZ_RMS: rms(sn.u_ss[f - KW_FIELD_UX_RMS]); return;
        case KW_FIELD_UX_FINAL: case KW_FIELD_UY_FINAL: case KW_FIELD_UZ_FINAL:
            d2h(h.dev.u[f - KW_FIELD_UX_FINAL], dst, (size_t)h.N);
            break;
        case KW_FIELD_IX_AVG: case KW_FIELD_IY_AVG: case KW_FIELD_IZ_AVG: {
            // intensityAvg (REC:113-124) with the half-sample shift kernel h[m] in FP64
            const int a = f - KW_FIELD_IX_AVG;
            if ((size_t)T * sizeof(float) > 200 * 1024) throw err(KW_ERR_UNSUPPORTED, "iAvg needs nt <= 51200");
            std::vector<double> hk(T, 0.0);
            const int half = T / 2;
            for (int m = 0; m < T; ++m) {
                double acc = 0;
                for (int k = 0; k < T; ++k) {
                    const int kk = k <= half ? k : k - T;
                    const double th = 2.0 * M_PI * (double)kk / (double)T * 0.5;
                    acc += std::cos(th + 2.0 * M_PI * (double)k * (double)m / (double)T);
                }
                hk[m] = acc / (double)T;
            }
            std::vector<float> hf = to_f32(hk);
            float* dh = (float*)dalloc(hf.size() * sizeof(float));
            check(cudaMemcpyAsync(dh, hf.data(), hf.size() * sizeof(float), cudaMemcpyHostToDevice, st()), "upload");
            float* out = (float*)dalloc(np * sizeof(float));
            launch_intensity(st(), sn.p_series, sn.u_series[a], T, (int)np, dh, out);
            check(cudaGetLastError(), "intensity");
            d2h(out, dst, np);
            break;
        }
        default: throw err(KW_ERR_INVALID, "unknown output field");
    }
    check(cudaStreamSynchronize(st()), "output sync");
}

}  // namespace kw
