// kw_adjoint.cpp — host orchestration of the discrete adjoint (equations in kw_adjoint.cu).
//
// 1. Forward run of the simulation (sensor p recorded), storing a checkpoint of the state after
//    every `interval`-th step (u_a, rho_a, S, p, div and S of the step before), or, with
//    KW_CHECKPOINT_STORE_ALL, the reverse sweep's inputs of every step.
// 2. Residuals r_t = p_sensor(t) - data(t) and the misfit on the host (FP64).
// 3. Reverse sweep, segment by segment from the last: restore the segment's checkpoint, rerun its
//    steps storing p, S, div (Stokes) and d_a = D-_a u_a (B/A; the density epilogue stores it) of
//    each step, then walk the segment backwards through the reverse step. The spectral pieces of
//    a reverse step are ordinary jobs of the pass kernels on FS_ADJ fields (the transposed
//    absorption filters with A2(S(t)), the source filter), and D+_a, D-_a whose C2R epilogues carry
//    the velocity adjoint and the sum into lambda_p (register row kernels; separate kernels
//    otherwise).
// 4. The t = 0 override of an initial pressure gives dL/dp0 and its share of dL/dc0.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <initializer_list>
#include <utility>
#include <vector>

#include "kw_adjoint.h"

#include <functional>
#include <map>
#include "kw_engine.h"

namespace kw {

static KwError err(int code, const std::string& m) { return KwError{code, m}; }

// Binomial checkpointing (Griewank's treeverse): with s free snapshot slots and the state before a
// stretch held, l steps are reversed with each step recomputed at most r times, r the least with
// beta(s, r) = C(s + r, s) >= l. A stretch is split at m: the states up to m are advanced once and
// the right part (l - m steps, s - 1 slots) needs l - m <= beta(s - 1, r), the left part (m steps,
// s slots, one repetition used) m <= beta(s, r - 1); any m between keeps the bound, the midpoint
// is taken.
static double binom_beta(int s, int r) {
    if (s < 0 || r < 0) return 0.0;
    double b = 1.0;   // C(s + r, s), capped far above any step count
    for (int i = 1; i <= r && b < 1e15; ++i) b = b * (s + i) / i;
    return b;
}
static int binom_reps(int l, int s) {
    int r = 0;
    while (binom_beta(s, r) < l) ++r;
    return r;
}
static int binom_split(int l, int s) {
    const int r = binom_reps(l, s);
    const int lo = std::max(1, (int)std::max(1.0, l - binom_beta(s - 1, r)));
    const int hi = (int)std::min((double)(l - 1), binom_beta(s, r - 1));
    return hi < lo ? lo : (lo + hi) / 2;
}
void Engine::adjoint(const kw_sim_desc& din, kw_adjoint_desc& a) {
    if (a.abi_version != KW_ABI_VERSION) throw err(KW_ERR_INVALID, "adjoint descriptor abi_version mismatch");
    if (!a.data) throw err(KW_ERR_INVALID, "adjoint: data is required");
    if (din.u_mask) throw err(KW_ERR_UNSUPPORTED, "adjoint: velocity sources are not supported");
    if (din.p_mask && din.p.data && din.p_mode != KW_SOURCE_ADDITIVE)
        throw err(KW_ERR_UNSUPPORTED, "adjoint: only the k-space corrected additive pressure source is supported");
    if (din.directivity_angle) throw err(KW_ERR_UNSUPPORTED, "adjoint: directivity is not supported");
    if (din.axisymmetric) throw err(KW_ERR_UNSUPPORTED, "adjoint: the axisymmetric solver is not supported");
    if ((din.smooth_c0 && din.sound_speed.len > 1) || (din.smooth_rho0 && din.density.len > 1))
        throw err(KW_ERR_UNSUPPORTED, "adjoint: smoothC0 / smoothRho0 maps are not supported");
    if (a.grad_p0 && !din.p0) throw err(KW_ERR_INVALID, "adjoint: grad_p0 needs source.p0");
    if (a.grad_p0 && din.smooth_p0) throw err(KW_ERR_UNSUPPORTED, "adjoint: grad_p0 with smoothP0 is not supported");
    const bool grho = a.grad_rho0 != nullptr;
    if (din.sensor_kind != KW_SENSOR_BINARY && din.sensor_kind != KW_SENSOR_CARTESIAN)
        throw err(KW_ERR_INVALID, "adjoint: a sensor is required");
    kw_sim_desc d = din;
    d.record = KW_RECORD_P;   // the reverse sweep reads the p series only
    precorrect_ok_ = false;   // the tape epilogues follow the per-step source job
    create(&d, 1);
    SimHost& h = sims_[0];
    SimDev& v = h.dev;
    const int D = h.dim, nt = h.nt;
    const long long N = h.N;
    const size_t fb = (size_t)N * sizeof(float);
    const int npts = v.sensor.npts;
    if (npts <= 0) throw err(KW_ERR_INVALID, "adjoint: the sensor has no points");
    const bool powerlaw = v.absorb >= 2, disp = v.absorb == 3, nonlin = v.nonlinear != 0;
    const bool has_p0 = v.has_p0 != 0;
    const bool psrc = v.has_p && v.psrc.mode == KW_SOURCE_ADDITIVE;
    float y = std::isnan(d.alpha_power) ? 1.5f : (float)d.alpha_power;
    if (d.alpha_mode == KW_ABSORPTION_STOKES) y = 2.f;

    // ---- work fields ----
    for (int k = 0; k < ADJ_COUNT; ++k)
        if (!adj_is_view(k) && (grho || k < ADJ_GP || k >= ADJ_GP + 3)) v.adj[k] = (float*)dalloc(fb);
    // the absorption job of the reverse step has three components, so it needs three spectra
    // (a 1D simulation allocates two)
    for (int k = 0; k < 3; ++k)
        if (!v.spec[k]) v.spec[k] = (float2*)dalloc((size_t)h.Ns * sizeof(float2));
    // the register row kernels fuse the velocity-adjoint and summing steps into their epilogues
    const bool fused = h.C % 2 == 0 && has_reg_row(h.M);
    // Folding the reverse equation of state into the absorption job's C2R saves its field traffic
    // on large grids; on small (L2-resident, launch-bound) grids the separate elementwise kernel
    // runs on more threads and is faster (2D 512^2: 3.13x against 3.24x forward time).
    // KW_ADJOINT_FUSED_EOS=1 / 0 forces the choice.
    // the summing step's operator pass adds up the components' spectra (register column kernel)
    const int last_n = D == 3 ? h.A : h.B;
    bool fanin = fused && D >= 2 && has_fixed_kernel(last_n) && has_colop(last_n);
    if (const char* f = std::getenv("KW_ADJOINT_FANIN")) fanin = fanin && f[0] == '1';
    bool eos_fused = N >= (1LL << 22);
    if (const char* f = std::getenv("KW_ADJOINT_FUSED_EOS")) eos_fused = f[0] == '1';
    double* gc = (double*)dalloc((size_t)N * sizeof(double));
    int* d_rev = (int*)dalloc(sizeof(int));
    v.adj_gc = gc;
    v.adj_rev = d_rev;
    v.adj_y = y;
    // density gradient: the direct terms and dL/d(dt / rho_sg_a), accumulated in FP64
    if (grho) {
        v.adj_gr = (double*)dalloc((size_t)N * sizeof(double));
        for (int b = 0; b < D; ++b) v.adj_gdtor[b] = (double*)dalloc((size_t)N * sizeof(double));
    }
    const bool keep_dd = nonlin || grho;   // the tape keeps d_a = D-_a u_a
    check(cudaMemcpyAsync(d_sims_, &v, sizeof(SimDev), cudaMemcpyHostToDevice, st()), "upload sim");

    // ---- checkpoint policy ----
    const bool stokes = v.absorb == 1;   // the Stokes term reads div(t); the power law only p(t), S(t)
    const int ck_fields = 2 * D + 3 + (stokes ? 1 : 0) + (grho ? 1 : 0);   // u_a, rho_a, S, p, S(t-1), div, p(t-1)
    const int CK_PPREV = 2 * D + 3 + (stokes ? 1 : 0);
    const int tp_fields = 2 + (stokes ? 1 : 0) + (keep_dd ? D : 0) + (disp ? 1 : 0);   // p, S, div, d_a, A2(S)
    bool store_all = a.policy == KW_CHECKPOINT_STORE_ALL;
    bool revolve = a.policy == KW_CHECKPOINT_REVOLVE;
    int nsnap = 0;   // revolve: snapshot slots (the held base state included)
    const double ck_bytes = (double)ck_fields * fb, tp_bytes = (double)tp_fields * fb;
    auto snaps_in = [&](double budget) { return (int)std::floor((budget - tp_bytes - 2.0 * fb) / ck_bytes); };
    // With checkpoints, segment c's recompute runs on the library's stream while segment c + 1 is
    // reversed on a second stream (the reverse sweep has its own spectra). The K tape slots are
    // walked forwards by even segments and backwards by odd ones, so the recompute of segment c
    // fills the slots in the order the reverse of segment c + 1 releases them; each recomputed step
    // waits for its slot's release. KW_ADJOINT_OVERLAP=0 runs them one after the other.
    bool overlap = true;
    if (const char* f = std::getenv("KW_ADJOINT_OVERLAP")) overlap = f[0] != '0';
    int K = 1;
    if (a.policy == KW_CHECKPOINT_SQRT) K = (int)std::ceil(std::sqrt((double)nt));
    else if (a.policy == KW_CHECKPOINT_INTERVAL) K = a.checkpoint_interval;
    else if (a.policy == KW_CHECKPOINT_BUDGET) {
        const double all = (double)nt * tp_fields * fb;
        if (all <= a.memory_budget) store_all = true;
        else {
            // memory(K) = ceil(nt / K) checkpoints + K tape slots
            double best = 1e300;
            for (int k = 1; k <= nt; ++k) {
                const double m = (double)((nt + k - 1) / k) * ck_fields * fb + (double)k * tp_fields * fb;
                if (m < best) { best = m; K = k; }
            }
            if (best > a.memory_budget) {   // no uniform interval fits: the binomial schedule
                revolve = true;
                nsnap = snaps_in(a.memory_budget);
                if (nsnap < 1)
                    throw err(KW_ERR_OOM, "adjoint: one state snapshot and one tape slot need more than memory_budget");
            }
        }
    } else if (revolve) {
        nsnap = a.checkpoint_interval > 0 ? a.checkpoint_interval : snaps_in(a.memory_budget);
        if (nsnap < 1) throw err(KW_ERR_OOM, "adjoint: one state snapshot and one tape slot need more than memory_budget");
    } else if (!store_all) throw err(KW_ERR_INVALID, "adjoint: unknown checkpoint policy");
    if (revolve) {
        nsnap = std::min(nsnap, nt);   // more slots than steps are never used
        K = 1;
        overlap = false;
    }
    if (store_all) K = nt;
    if (K < 1 || K > nt) throw err(KW_ERR_INVALID, "adjoint: checkpoint_interval must be in [1, nt]");
    const int nck = revolve ? nsnap : (store_all ? 0 : (nt + K - 1) / K);
    if (nck < 2) overlap = false;
    a.interval = revolve ? 0 : K;
    a.checkpoints = nck;

    // tape: K slots of tp_fields fields; checkpoints: nck of ck_fields fields
    auto alloc_fields = [&](size_t count) {
        std::vector<float*> f(count);
        for (auto& x : f) x = (float*)dalloc(fb);
        return f;
    };
    std::vector<float*> tape = alloc_fields((size_t)K * tp_fields);
    std::vector<float*> ck = alloc_fields((size_t)nck * ck_fields);
    auto tslot = [&](int slot, int f) { return tape[(size_t)slot * tp_fields + f]; };   // f: 0 p, 1 S, 2 div, then d_a, A2(S)
    const int TF_DIV = 2, TF_DD = stokes ? 3 : 2, TF_Q2 = TF_DD + (keep_dd ? D : 0);
    auto ckf = [&](int c, int f) { return ck[(size_t)c * ck_fields + f]; };   // u_a, rho_a, S, p, S(t-1), div
    auto cpy = [&](float* dst, const float* src) {
        check(cudaMemcpyAsync(dst, src, fb, cudaMemcpyDeviceToDevice, st()), "adjoint copy");
    };
    auto zero = [&](float* x) { check(cudaMemsetAsync(x, 0, fb, st()), "adjoint zero"); };
    float* zero_field = (float*)dalloc(fb);   // S(-1): the state before step 0 is zero
    // revolve: S(t-1) and p(t-1) of the step whose tape the single slot holds
    float* rv_sprev = revolve ? (float*)dalloc(fb) : nullptr;
    float* rv_pprev = revolve && grho ? (float*)dalloc(fb) : nullptr;

    // tape slot of step t: even segments walk the slots forwards, odd ones backwards
    auto slot_of = [&](int t) { return store_all ? t : ((t / K) % 2 == 0 ? t % K : K - 1 - t % K); };
    // where step t's forward quantities live while the reverse sweep reads them
    std::vector<AdjTapeEntry> table(nt);
    for (int t = 0; t < nt; ++t) {
        const int slot = slot_of(t);
        AdjTapeEntry& e = table[t];
        e.p = tslot(slot, 0);
        e.s = tslot(slot, 1);
        e.div = stokes ? tslot(slot, TF_DIV) : nullptr;
        for (int b = 0; b < kMaxComp; ++b) e.dd[b] = keep_dd && b < D ? tslot(slot, TF_DD + b) : nullptr;
        e.q2 = disp ? tslot(slot, TF_Q2) : nullptr;
        e.pprev = !grho ? nullptr
                        : (t == 0 ? zero_field : (store_all || t % K > 0 ? tslot(slot_of(t - 1), 0) : ckf(t / K, CK_PPREV)));
        e.sprev = t == 0 ? zero_field : (store_all || t % K > 0 ? tslot(slot_of(t - 1), 1) : ckf(t / K, 2 * D + 2));
        if (revolve && t > 0) {
            e.sprev = rv_sprev;
            if (grho) e.pprev = rv_pprev;
        }
    }
    const AdjTapeEntry* d_table = upload(table);
    v.tape = d_table;
    check(cudaMemcpyAsync(d_sims_, &v, sizeof(SimDev), cudaMemcpyHostToDevice, st()), "upload sim");
    // Steps captured in tape mode store p, S, div, d_a and A2(S) of step t into table[t] from their
    // epilogues; a restored checkpoint (and step 0, whose t = 0 override follows its epilogues) is
    // copied into its slot instead.
    auto tape_copy = [&]() { launch_adj_tape(st(), d_sims_, d_t_, d_table, stokes, N); };
    auto set_tape_mode = [&](bool on) {
        tape_mode_ = on;
        for (int g = 0; g < 2; ++g) {
            if (graph_exec_[g]) { cudaGraphExecDestroy(graph_exec_[g]); graph_exec_[g] = nullptr; }
            if (graph_[g]) { cudaGraphDestroy(graph_[g]); graph_[g] = nullptr; }
        }
    };

    cudaEvent_t e0, e1, e2;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    check(cudaEventCreate(&e2), "event");

    // ---- 1. forward ----
    // The last segment (every step with store-all) fills the tape as it runs, so the reverse sweep
    // starts with its reverse instead of recomputing it.
    const int t_last = revolve ? nt : (store_all ? 0 : (nck - 1) * K);
    set_tape_mode(t_last == 0);
    reset();
    // revolve: the residual sweep stores the snapshots of the schedule's right spine (the base state
    // of the reversed steps, then each first split of the remaining stretch with one slot fewer)
    const int t_stop = has_p0 ? 1 : 0;
    std::map<int, int> spine;   // step t -> snapshot slot holding the state after step t
    if (revolve) {
        int lo = t_stop, s_free = nsnap - 1;
        spine[lo] = 0;
        while (nt - lo > 1 && s_free > 0) {
            lo += binom_split(nt - lo, s_free);
            spine[lo] = nsnap - s_free;
            --s_free;
        }
    }
    check(cudaEventRecord(e0, st()), "event");
    for (int t = 0; t < nt; ++t) {
        const bool ck_step = revolve ? spine.count(t) > 0 : (!store_all && t % K == 0);
        if (ck_step) {
            const int c = revolve ? spine[t] : t / K;
            if (t == 0) zero(ckf(c, 2 * D + 2));
            else cpy(ckf(c, 2 * D + 2), v.rho_sum);
            if (grho) {
                if (t == 0) zero(ckf(c, CK_PPREV));
                else cpy(ckf(c, CK_PPREV), v.p);
            }
        }
        if (t == t_last && !tape_mode_) set_tape_mode(true);
        step(1);
        if (tape_mode_ && t == 0) tape_copy();   // the t = 0 override follows the step's epilogues
        if (ck_step) {
            const int c = revolve ? spine[t] : t / K;
            for (int b = 0; b < D; ++b) { cpy(ckf(c, b), v.u[b]); cpy(ckf(c, D + b), v.rho[b]); }
            cpy(ckf(c, 2 * D), v.rho_sum);
            cpy(ckf(c, 2 * D + 1), v.p);
            if (stokes) cpy(ckf(c, 2 * D + 3), v.div_term);
        }
    }
    check(cudaEventRecord(e1, st()), "event");

    // ---- 2. residuals and misfit ----
    std::vector<float> ps((size_t)nt * npts);
    check(cudaMemcpyAsync(ps.data(), v.sensor.p_series, ps.size() * sizeof(float), cudaMemcpyDeviceToHost, st()), "series");
    check(cudaStreamSynchronize(st()), "sync");
    check_kernel_error();
    std::vector<float> resid((size_t)nt * npts);   // [t][q]
    double L = 0;
    for (int t = 0; t < nt; ++t)
        for (int q = 0; q < npts; ++q) {
            const double r = (double)ps[(size_t)t * npts + q] - (double)a.data[(size_t)q * nt + t];
            resid[(size_t)t * npts + q] = (float)r;
            L += 0.5 * r * r;
        }
    a.misfit = L;
    float* d_resid = upload(resid);

    // ---- 3. reverse sweep ----
    // the recomputed segments do not sample the sensor and fill the tape: capture the forward step
    // again that way
    any_recp_ = false;
    set_tape_mode(true);
    for (int k = 0; k < ADJ_COUNT; ++k)
        if (!adj_is_view(k) && v.adj[k]) zero(v.adj[k]);
    check(cudaMemsetAsync(gc, 0, (size_t)N * sizeof(double), st()), "zero");
    if (grho) {
        check(cudaMemsetAsync(v.adj_gr, 0, (size_t)N * sizeof(double), st()), "zero");
        for (int b = 0; b < D; ++b) check(cudaMemsetAsync(v.adj_gdtor[b], 0, (size_t)N * sizeof(double), st()), "zero");
    }

    // The overlapped sweep: the reverse steps are issued on their own stream against a copy of the
    // simulation descriptor with its own spectra (and tensor maps), step counter and tape views.
    const cudaStream_t fs = st();
    cudaStream_t rs = nullptr;
    SimDev* d_sims_rev = nullptr;
    int* d_t_rev = nullptr;
    cudaEvent_t ev_rec = nullptr, ev_done = nullptr;
    std::vector<cudaEvent_t> ev_free;   // per tape slot: its last reader in the reverse sweep is done
    if (overlap) {
        SimDev vr = v;
        for (int k = 0; k < 4; ++k) {
            vr.spec[k] = nullptr;
            if (v.spec[k]) {
                vr.spec[k] = (float2*)dalloc((size_t)h.Ns * sizeof(float2));
                check(cudaMemsetAsync(vr.spec[k], 0, (size_t)h.Ns * sizeof(float2), fs), "zero");
            }
        }
        vr.tmaps = nullptr;
        build_tensor_maps(h, vr);
        d_sims_rev = (SimDev*)dalloc(sizeof(SimDev));
        check(cudaMemcpyAsync(d_sims_rev, &vr, sizeof(SimDev), cudaMemcpyHostToDevice, fs), "upload sim");
        d_t_rev = (int*)dalloc(sizeof(int));
        check(cudaStreamCreateWithFlags(&rs, cudaStreamNonBlocking), "stream");
        for (cudaEvent_t* e : {&ev_rec, &ev_done})
            check(cudaEventCreateWithFlags(e, cudaEventDisableTiming), "event");
        ev_free.assign(K, nullptr);
        for (auto& e : ev_free) {
            check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
            check(cudaEventRecord(e, fs), "event");   // every slot is free
        }
        // the reverse stream starts after the zeroing above
        check(cudaEventRecord(ev_rec, fs), "event");
        check(cudaStreamWaitEvent(rs, ev_rec, 0), "wait");
    }
    // issue `fn` as reverse-sweep work (on the reverse stream when overlapped)
    auto on_reverse = [&](auto&& fn) {
        if (!overlap) { fn(); return; }
        std::swap(d_sims_, d_sims_rev);
        std::swap(d_t_, d_t_rev);
        st_override_ = rs;
        auto back = [&] {
            std::swap(d_sims_, d_sims_rev);
            std::swap(d_t_, d_t_rev);
            st_override_ = nullptr;
        };
        try {
            fn();
        } catch (...) {
            back();
            throw;
        }
        back();
    };
    AdjStepArgs A{};
    A.a1 = v.adj[ADJ_A1];
    A.a2 = v.adj[ADJ_A2];
    A.lam_p = v.adj[ADJ_LP];
    for (int b = 0; b < kMaxComp; ++b) {
        const int bb = b < D ? b : 0;
        A.lam_u[b] = v.adj[ADJ_LU + bb];
        A.lam_r[b] = v.adj[ADJ_LR + bb];
        A.w[b] = v.adj[ADJ_W + bb];
        A.e[b] = v.adj[ADJ_E + bb];
    }
    A.gc = gc;
    A.y = y;

    // fwd_spec / r2c_done: row fusion (the adjoint velocity C2R transforms the new w_a into the
    // summing job's input spectra, kw_jobs.cpp)
    auto job_in = [&](int in_field, int out, int nin, auto opf, int epi, int coupled, const char* name, int fanin = 0,
                      int fwd_spec = -1, int r2c_done = 0) {
        SpecJob j;
        j.fwd_spec = fwd_spec;
        j.r2c_done = r2c_done;
        j.in_field = in_field;
        j.nin = nin;
        j.nout = fanin ? 1 : nin;
        j.fanin = fanin ? nin : 0;
        for (int c = 0; c < nin; ++c) j.op[c] = opf(c);
        j.spec_in = 0;
        j.spec_out = 0;
        j.epi = epi;
        j.coupled = coupled;
        j.out_field = FS_ADJ + out;
        j.name = name;
        issue_job(j, -1);
    };
    auto job = [&](int in, int out, int nin, auto opf, int epi, int coupled, const char* name, int fanin = 0,
                   int fwd_spec = -1, int r2c_done = 0) {
        job_in(FS_ADJ + in, out, nin, opf, epi, coupled, name, fanin, fwd_spec, r2c_done);
    };
    const bool fuse_w = D >= 2 && fuse_rows();
    // absorption filters: x1 with |k|^(y-2); x2 with |k|^(y-1) (A2(S(t)) comes from the tape)
    auto absorption_op = [](int c) { return OpSpec{AO_NONE, 0, (int8_t)(c == 0 ? RT_NU1 : RT_NU2), (int8_t)c}; };
    auto radial = [](int r) { return [r](int c) { return OpSpec{AO_NONE, 0, (int8_t)r, (int8_t)c}; }; };
    auto deriv = [](int ao) { return [ao](int c) { return OpSpec{(int8_t)ao, (int8_t)c, RT_KAPPA, (int8_t)c}; }; };

    // one reverse step; its step t comes from *d_rev (counted down), so the launches are the same
    // for every step and run as a CUDA graph (one per variant: additive source active or not)
    auto reverse_body = [&](bool src_on) {
        launch_adj_begin(st(), d_sims_, d_t_, d_rev, d_table, d_resid, npts);   // also sets the step counter the pass kernels gate on
        A.sig = src_on ? v.adj[ADJ_SIG] : nullptr;
        if (powerlaw && fused && eos_fused) {   // the absorption filters with the reverse EoS as epilogue
            job(ADJ_X1, ADJ_A1, disp ? 2 : 1, absorption_op, grho ? EPI_ADJ_EOS_RHO : EPI_ADJ_EOS, 1, "adj_eos");
        } else {
            if (powerlaw) job(ADJ_X1, ADJ_A1, disp ? 2 : 1, absorption_op, EPI_STORE, 0, "adj_abs");
            launch_adj_eos(st(), d_sims_, N, A, d_rev, grho);
        }
        if (src_on) {
            job(ADJ_SIG, ADJ_GSIG, 1, radial(RT_SKAPPA), EPI_STORE, 0, "adj_src");
            launch_adj_src(st(), d_sims_, v.psrc.nsrc, v.adj[ADJ_GSIG], d_t_, gc);
        }
        if (grho) {   // g_a = D+_a p(t-1) of the velocity update, for dL/d(dt / rho_sg_a)
            SpecJob gj;
            gj.in_field = FS_ADJ + ADJ_PPREV;
            gj.nin = 1;
            gj.fanout = 1;
            gj.nout = D;
            for (int b = 0; b < D; ++b) gj.op[b] = OpSpec{AO_DPOS, (int8_t)b, RT_KAPPA, 0};
            gj.epi = EPI_STORE;
            gj.out_field = FS_ADJ + ADJ_GP;
            gj.name = "adj_gp";
            issue_job(gj, -1);
        }
        if (fused) {
            job(ADJ_W, ADJ_E, D, deriv(AO_DPOS), grho ? EPI_ADJ_VEL_RHO : EPI_ADJ_VEL, 0, "adj_vel", 0, fuse_w ? 0 : -1);
            // lambda_p = sum_a D-_a w_a: the operator pass sums the components' spectra, so one
            // inverse transform serves all of them
            job(ADJ_W, ADJ_E, D, deriv(AO_DNEG), EPI_ADJ_SUM, 1, "adj_sum", fanin ? 1 : 0, -1, fuse_w ? 1 : 0);
        } else {
            job(ADJ_W, ADJ_E, D, deriv(AO_DPOS), EPI_STORE, 0, "adj_dpos");
            launch_adj_vel(st(), d_sims_, N, A);
            job(ADJ_W, ADJ_E, D, deriv(AO_DNEG), EPI_STORE, 0, "adj_dneg");
            launch_adj_sum(st(), d_sims_, N, A);
        }
    };
    cudaGraphExec_t rgraph[2] = {nullptr, nullptr};
    int uses[2] = {0, 0};
    auto reverse_step = [&](int t) {
        const int var = psrc && t < v.psrc.len ? 1 : 0;
        if (uses[var]++ == 0) {   // the first use runs directly (it also creates the tile maps)
            reverse_body(var == 1);
            return;
        }
        if (!rgraph[var]) {
            cudaGraph_t g = nullptr;
            check(cudaStreamBeginCapture(st(), cudaStreamCaptureModeThreadLocal), "begin capture");
            try {
                reverse_body(var == 1);
            } catch (...) {
                cudaStreamEndCapture(st(), &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            check(cudaStreamEndCapture(st(), &g), "end capture");
            const cudaError_t e = cudaGraphInstantiate(&rgraph[var], g, 0);
            cudaGraphDestroy(g);
            check(e, "graph instantiate");
        }
        check(cudaGraphLaunch(rgraph[var], st()), "graph launch");
    };

    on_reverse([&] { launch_set_step(st(), d_rev, nt - 1); });
    if (revolve) {
        // snapshot c holds the state after some step t (u, rho, S, p, div) and S(t-1), p(t-1)
        set_tape_mode(false);
        std::vector<int> free_slots;
        for (int c = nsnap - 1; c >= 1; --c) {
            bool used = false;
            for (auto& kv : spine) used = used || kv.second == c;
            if (!used) free_slots.push_back(c);
        }
        auto restore = [&](int c, int t) {   // the state after step t, from snapshot c
            for (int b = 0; b < D; ++b) { cpy(v.u[b], ckf(c, b)); cpy(v.rho[b], ckf(c, D + b)); }
            cpy(v.rho_sum, ckf(c, 2 * D));
            cpy(v.p, ckf(c, 2 * D + 1));
            if (stokes) cpy(v.div_term, ckf(c, 2 * D + 3));
            launch_set_step(st(), d_t_, t + 1);
            t_ = t + 1;
        };
        // advance from the state after step a (snapshot ca) to the state after step m; with
        // cm >= 0 store it in snapshot cm, else leave it live with S(m-1), p(m-1) in rv_sprev / rv_pprev
        auto advance = [&](int ca, int a0, int m, int cm) {
            restore(ca, a0);
            for (int t = a0 + 1; t <= m; ++t) {
                if (t == m) {
                    cpy(cm >= 0 ? ckf(cm, 2 * D + 2) : rv_sprev, v.rho_sum);
                    if (grho) cpy(cm >= 0 ? ckf(cm, CK_PPREV) : rv_pprev, v.p);
                }
                step(1);
            }
            if (cm >= 0) {
                for (int b = 0; b < D; ++b) { cpy(ckf(cm, b), v.u[b]); cpy(ckf(cm, D + b), v.rho[b]); }
                cpy(ckf(cm, 2 * D), v.rho_sum);
                cpy(ckf(cm, 2 * D + 1), v.p);
                if (stokes) cpy(ckf(cm, 2 * D + 3), v.div_term);
            }
        };
        // the tape of step t from the live state after step t (S(t-1), p(t-1) already in place)
        auto tape_live = [&](int t) {
            if (keep_dd || disp) {
                launch_set_step(st(), d_t_, t);
                launch_adj_views(st(), d_sims_, d_table, t);
                if (keep_dd) job_in(FS_U, ADJ_DDP, D, deriv(AO_DNEG), EPI_STORE, 0, "adj_du");
                if (disp) job_in(FS_RHO_SUM, ADJ_Q2, 1, radial(RT_NU2), EPI_STORE, 0, "adj_q2");
            }
            launch_set_step(st(), d_t_, t + 1);
            t_ = t + 1;
            tape_copy();
        };
        auto tape_from = [&](int c, int t) {
            restore(c, t);
            if (t > 0) {
                cpy(rv_sprev, ckf(c, 2 * D + 2));
                if (grho) cpy(rv_pprev, ckf(c, CK_PPREV));
            }
            tape_live(t);
        };
        // reverse steps b, b-1, ..., a with the state after step a in snapshot ca and s free slots
        std::function<void(int, int, int, int)> rev = [&](int a0, int b, int s, int ca) {
            if (a0 == b) {
                tape_from(ca, a0);
                reverse_step(a0);
                return;
            }
            if (s == 0) {
                for (int t = b; t > a0; --t) {
                    advance(ca, a0, t, -1);
                    tape_live(t);
                    reverse_step(t);
                }
                tape_from(ca, a0);
                reverse_step(a0);
                return;
            }
            const int m = a0 + binom_split(b - a0 + 1, s);
            int cm;
            auto it = spine.find(m);
            if (it != spine.end() && it->first != t_stop) {
                cm = it->second;   // stored by the residual sweep
                spine.erase(it);
            } else {
                cm = free_slots.back();
                free_slots.pop_back();
                advance(ca, a0, m, cm);
            }
            rev(m, b, s - 1, cm);
            free_slots.push_back(cm);
            rev(a0, m - 1, s, ca);
        };
        if (nt - 1 >= t_stop) rev(t_stop, nt - 1, nsnap - 1, spine[t_stop]);
    } else if (store_all) {
        for (int t = nt - 1; t >= t_stop; --t) reverse_step(t);
    } else {
        for (int c = nck - 1; c >= 0; --c) {
            const int t0 = c * K, t1 = std::min(t0 + K, nt);
            if (t1 - 1 < t_stop) continue;
            // slot writes wait until the reverse of segment c + 1 has released the slot
            auto slot_free = [&](int t) {
                if (overlap) check(cudaStreamWaitEvent(fs, ev_free[slot_of(t)], 0), "wait");
            };
            // the last segment's tape is still in place from the forward
            if (c < nck - 1) {
                slot_free(t0);
                // restore the state after step t0 and rerun the segment, storing each step
                for (int b = 0; b < D; ++b) { cpy(v.u[b], ckf(c, b)); cpy(v.rho[b], ckf(c, D + b)); }
                cpy(v.rho_sum, ckf(c, 2 * D));
                cpy(v.p, ckf(c, 2 * D + 1));
                if (stokes) cpy(v.div_term, ckf(c, 2 * D + 3));
                if (keep_dd || disp) {   // d_a(t0) = D-_a u_a(t0), A2(S(t0)) of the restored state into its tape slot
                    launch_set_step(st(), d_t_, t0);
                    launch_adj_views(st(), d_sims_, d_table, t0);
                    if (keep_dd) job_in(FS_U, ADJ_DDP, D, deriv(AO_DNEG), EPI_STORE, 0, "adj_du");
                    if (disp) job_in(FS_RHO_SUM, ADJ_Q2, 1, radial(RT_NU2), EPI_STORE, 0, "adj_q2");
                }
                launch_set_step(st(), d_t_, t0 + 1);
                t_ = t0 + 1;
                tape_copy();
                for (int t = t0 + 1; t < t1; ++t) {
                    slot_free(t);
                    step(1);
                }
            }
            if (overlap) {
                check(cudaEventRecord(ev_rec, fs), "event");
                check(cudaStreamWaitEvent(rs, ev_rec, 0), "wait");
            }
            // the reverse of this segment overlaps the recompute of the next one
            on_reverse([&] {
                for (int t = t1 - 1; t >= std::max(t0, t_stop); --t) {
                    reverse_step(t);
                    if (overlap) check(cudaEventRecord(ev_free[slot_of(t)], rs), "event");
                }
            });
        }
        if (overlap) {
            check(cudaEventRecord(ev_done, rs), "event");
            check(cudaStreamWaitEvent(fs, ev_done, 0), "wait");
        }
    }
    if (has_p0) {
        // t = 0 override: p = p0, rho_a = p0 / (D c^2), u_a = dtor_a / 2 D+_a p0
        launch_adj_begin(st(), d_sims_, d_t_, d_rev, d_table, d_resid, npts);   // *d_rev is 0 here: residual r_0
        if (grho) {   // u_a = dtor_a / 2 D+_a p0: g_a = D+_a p0 into ADJ_GP, then dL/d dtor_a += lambda_u_a g_a / 2
            check(cudaMemcpyAsync(v.adj[ADJ_GP], h.p0s, fb, cudaMemcpyDeviceToDevice, st()), "p0 copy");
            SpecJob gj;
            gj.in_field = FS_ADJ + ADJ_GP;
            gj.nin = 1;
            gj.fanout = 1;
            gj.nout = D;
            for (int b = 0; b < D; ++b) gj.op[b] = OpSpec{AO_DPOS, (int8_t)b, RT_KAPPA, 0};
            gj.epi = EPI_STORE;
            gj.out_field = FS_ADJ + ADJ_GP;
            gj.name = "adj_gp0";
            issue_job(gj, -1);
            launch_adj_rho_p0(st(), d_sims_, N);
        }
        launch_adj_half_dtor(st(), d_sims_, N, A);
        job(ADJ_W, ADJ_E, D, deriv(AO_DNEG), EPI_STORE, 0, "adj_p0");
        float* gp = a.grad_p0 ? v.adj[ADJ_GSIG] : nullptr;
        launch_adj_p0(st(), d_sims_, N, A, h.p0s, gp);
        if (gp) {
            check(cudaMemcpyAsync(a.grad_p0, gp, fb, cudaMemcpyDeviceToHost, st()), "grad p0");
        }
    } else if (a.grad_p0) {
        std::memset(a.grad_p0, 0, fb);
    }
    check(cudaEventRecord(e2, st()), "event");
    if (a.grad_c0) {
        launch_adj_store_grad(st(), gc, v.adj[ADJ_SIG], N);
        check(cudaMemcpyAsync(a.grad_c0, v.adj[ADJ_SIG], fb, cudaMemcpyDeviceToHost, st()), "grad c0");
    }
    if (grho) {
        launch_adj_rho_final(st(), d_sims_, N, v.adj[ADJ_GSIG]);
        check(cudaMemcpyAsync(a.grad_rho0, v.adj[ADJ_GSIG], fb, cudaMemcpyDeviceToHost, st()), "grad rho0");
    }
    check(cudaGetLastError(), "adjoint launch");
    check(cudaStreamSynchronize(st()), "adjoint sync");
    check_kernel_error();
    float f_ms = 0, r_ms = 0;
    cudaEventElapsedTime(&f_ms, e0, e1);
    cudaEventElapsedTime(&r_ms, e1, e2);
    a.forward_ms = f_ms;
    a.reverse_ms = r_ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    for (auto& g : rgraph)
        if (g) cudaGraphExecDestroy(g);
    if (rs) {
        cudaStreamSynchronize(rs);
        cudaStreamDestroy(rs);
        for (cudaEvent_t e : {ev_rec, ev_done})
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : ev_free)
            if (e) cudaEventDestroy(e);
    }
    set_tape_mode(false);
    v.tape = nullptr;
    check(cudaMemcpyAsync(d_sims_, &v, sizeof(SimDev), cudaMemcpyHostToDevice, st()), "upload sim");
}

}  // namespace kw
