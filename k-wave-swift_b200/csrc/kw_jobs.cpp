// kw_jobs.cpp — tile maps and the launch sequence of one spectral job:
//   R2C rows -> column passes (the k-space operator fused into the last) -> C2R rows + epilogue.
// Each pass is launched once per size class (line length) of the engine's simulations, so every
// launch runs the kernel instantiation specialised for its line length.
#include "kw_engine.h"

#include <algorithm>
#include <cstdlib>
#include <set>

namespace kw {

// size class of a row pass / column pass of one simulation (0 = runtime-plan kernels)
static int row_class(const SimHost& h) {
    return (h.C % 2 == 0 && (has_fixed_kernel(h.M) || has_reg_row(h.M))) ? h.M : 0;
}
// register-resident row kernels (kw_pass_rowr.cu) serve the even rows of two-stage half length;
// the 1D forward row pass, which also applies the operator, keeps the staged kernel
static bool rowr_class(int sclass) { return sclass != 0 && has_reg_row(sclass); }
// which register column kernels run: bit 0 the operator pass on the double-buffered kernel (else
// one tile per CTA), bit 1 the in-place passes up to 256 points on it too (else TMA-fed), bit 2
// the in-place passes above 256 points on the staged kernels (else double-buffered); KW_COLA
// overrides
static int cola_policy() {
    if (const char* e = std::getenv("KW_COLA")) return std::atoi(e);
    return 0;
}
// the 3D R2C and forward pass along B as one cluster kernel per plane (kw_pass_plane.cu), opt-in
// with KW_PLANE=1: on a B200 at 256^3 it moves 1.8 TB/s of algorithmic bytes against 4.2 TB/s for
// the two separate passes (its phases serialise on the cluster barriers), so the separate passes
// are the default
static bool plane_policy() {
    if (const char* e = std::getenv("KW_PLANE")) return e[0] == '1';
    return false;
}
// Row fusion: the register C2R of a job also runs the forward R2C of its epilogue's output into
// the next job's input spectra (velocity -> density, density -> power-law absorption, adjoint
// velocity -> adjoint sum), so the next job skips its R2C and the field is not read back. Opt-in
// with KW_FUSE_ROWS=1: on a B200 at 256^3 the fused C2R kernels move 3.6 TB/s of algorithmic
// bytes against 4.6-4.7 TB/s for the separate C2R and R2C, and the step took 1.52 ms against
// 1.47 ms unfused, although it moves 8 % fewer bytes.
bool Engine::fuse_rows() const {
    if (plane_policy()) return false;
    const char* e = std::getenv("KW_FUSE_ROWS");
    return e && e[0] == '1';
}
// Traversal order of the tile maps. A pass reads what the previous one wrote, and the last part
// written (up to ~100 MB at 256^3) is still in L2 when the next kernel starts; CTAs are started
// in map order, so a pass over the same plane-major layout that walks its tiles the other way
// round starts on those lines. The R2C and the inverse pass along B walk forwards, the forward
// pass along B and the C2R backwards (the operator pass along A reads every plane in each tile
// and breaks the chain). KW_MAP_ORDER=0: every map forwards.
// KW_MAP_ORDER=2: the column passes walk column-chunk-major instead (forward pass along B
// forwards, operator pass backwards, inverse pass along B forwards), so the column-to-column
// transitions start on the resident lines rather than the row-to-column ones.
static int map_order_policy() {
    const char* e = std::getenv("KW_MAP_ORDER");
    return e ? std::atoi(e) : 1;
}
static bool alternate_order() { return map_order_policy() != 0; }

// The register R2C and the one-component C2R kernels also prefetch into L2 the rows of the CTA one
// resident wave on (the SM count times the resident CTAs per SM of the kernel). Measured at 256^3:
// R2C 3-5 % and the velocity C2R 5 % faster, while the coupled density and power-law C2R, which
// already prefetch their epilogues' fields, got 4-11 % slower with it, so those do not.
// KW_ROW_AHEAD=0 turns it off.
static int row_ahead(int per_sm) {
    const char* e = std::getenv("KW_ROW_AHEAD");
    if (e && e[0] == '0') return 0;
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            sms = 1;
        }
    }
    return sms * per_sm;
}

// KW_COLP_AHEAD=n: the TMA-fed in-place column pass also prefetches into L2 (one tensor prefetch)
// the tile n of its tiles on, beyond its two-stage ring; 0 (default): none
static int colp_ahead() {
    const char* e = std::getenv("KW_COLP_AHEAD");
    return e ? std::max(0, std::atoi(e)) : 0;
}

// bulk L2 prefetch of the C2R epilogue's field rows (k_rowr_c2r); KW_C2R_PREFETCH=0 turns it off
static bool c2r_prefetch() {
    const char* e = std::getenv("KW_C2R_PREFETCH");
    return !(e && e[0] == '0');
}
static int col_class(const SimHost& h, int axis) {
    const int n = axis == 0 ? h.A : h.B;
    return has_fixed_kernel(n) ? n : 0;
}

// Row-pass tiles of the simulations of size class `sclass`. lines_per_row == 0: R2C tiles of
// row_lines(M) rows; lines_per_row > 0: C2R tiles of c2r_lines(M) lines, i.e. c2r_lines(M) /
// lines_per_row rows (a coupled C2R epilogue stages every component of a row in the same CTA);
// lines_per_row = -1 / -2: tiles of r2c_rows(M) / c2r_rows(M) rows for the register-resident R2C /
// C2R kernels.
const Engine::Map& Engine::map_rows(int lines_per_row, int ncomp, int sim_only, int sclass, bool reverse) {
    auto key = std::make_tuple(reverse ? 20 : 0, lines_per_row, ncomp, sim_only, sclass);
    auto it = maps_.find(key);
    if (it != maps_.end()) return it->second;
    std::vector<BlockWork> v;
    for (int s = 0; s < count(); ++s) {
        if ((sim_only >= 0 && s != sim_only) || row_class(sims_[s]) != sclass) continue;
        const int rows = sims_[s].A * sims_[s].B;
        const int rpc = lines_per_row == -1  ? r2c_rows(sims_[s].M)
                        : lines_per_row == -2 ? c2r_rows(sims_[s].M)
                        : lines_per_row == 0  ? row_lines(sims_[s].M)
                                              : std::max(1, c2r_lines(sims_[s].M) / lines_per_row);
        const int tiles = (rows + rpc - 1) / rpc;
        for (int c = 0; c < ncomp; ++c)
            for (int tI = 0; tI < tiles; ++tI) v.push_back(BlockWork{s, c, tI});
    }
    if (reverse) std::reverse(v.begin(), v.end());
    Map m;
    m.d = upload(v);
    m.n = (int)v.size();
    return maps_[key] = m;
}

// Column-pass tiles: col_lines(n) (col_lines_op(n) for an operator pass) contiguous columns, or
// for the register-plan lengths colr_lines(n) (colop_lines(n)) columns of one plane.
const Engine::Map& Engine::map_cols(int axis, int ncomp, int sim_only, bool op, int sclass, int tw_op, int order) {
    auto key = std::make_tuple(1 + axis + (op ? 2 : 0) + 20 * order, tw_op, ncomp, sim_only, sclass);
    auto it = maps_.find(key);
    if (it != maps_.end()) return it->second;
    std::vector<BlockWork> v;
    for (int s = 0; s < count(); ++s) {
        if ((sim_only >= 0 && s != sim_only) || col_class(sims_[s], axis) != sclass) continue;
        const SimHost& h = sims_[s];
        const int n = axis == 0 ? h.A : h.B;
        const int inner = axis == 0 ? h.B * h.Cp : h.Cp;
        const int outer = axis == 0 ? 1 : h.A;
        int tiles, tw;
        const bool reg = op ? has_colop(sclass) : (has_colp(sclass) || (has_colop(sclass) && !(cola_policy() & 4)));
        if (sclass && reg) {   // register-plan kernels: columns of one plane
            tw = op ? (tw_op > 0 ? tw_op : colop_lines(n)) : colr_lines(n);
            tiles = outer * ((inner + tw - 1) / tw);
        } else {
            tw = op ? col_lines_op(n) : col_lines(n);
            tiles = outer * ((inner + tw - 1) / tw);
        }
        // tile order within a component: plane-major (as numbered), or for order 2 / 3 and the
        // register-plan kernels column-chunk-major (all planes / rows of one chunk of spectrum
        // bins together, chunks by their first bin)
        std::vector<int> seq(tiles);
        for (int tI = 0; tI < tiles; ++tI) seq[tI] = tI;
        if (order >= 2 && sclass && reg) {
            const int nch = (inner + tw - 1) / tw;
            auto rank = [&](int tI) -> long long {
                if (axis == 1) return (long long)(tI % nch) * outer + tI / nch;   // (chunk, plane)
                const int c0 = tI * tw;                                          // (bin, row of B)
                return (long long)(c0 % h.Cp) * h.B + c0 / h.Cp;
            };
            std::stable_sort(seq.begin(), seq.end(), [&](int x, int y) { return rank(x) < rank(y); });
        }
        for (int c = 0; c < ncomp; ++c)
            for (int tI : seq) v.push_back(BlockWork{s, c, tI});
    }
    if (order == 1 || order == 3) std::reverse(v.begin(), v.end());
    Map m;
    m.d = upload(v);
    m.n = (int)v.size();
    return maps_[key] = m;
}

// Plane-pass items: (simulation, component, plane a), components outer.
const Engine::Map& Engine::map_planes(int ncomp, int sim_only) {
    auto key = std::make_tuple(10, 0, ncomp, sim_only, 0);
    auto it = maps_.find(key);
    if (it != maps_.end()) return it->second;
    std::vector<BlockWork> v;
    for (int s = 0; s < count(); ++s) {
        if (sim_only >= 0 && s != sim_only) continue;
        for (int c = 0; c < ncomp; ++c)
            for (int a = 0; a < sims_[s].A; ++a) v.push_back(BlockWork{s, c, a});
    }
    Map m;
    m.d = upload(v);
    m.n = (int)v.size();
    return maps_[key] = m;
}

const Engine::Map& Engine::map_elems(int sim_only) {
    auto key = std::make_tuple(9, 0, 0, sim_only, 0);
    auto it = maps_.find(key);
    if (it != maps_.end()) return it->second;
    std::vector<BlockWork> v;
    for (int s = 0; s < count(); ++s) {
        if (sim_only >= 0 && s != sim_only) continue;
        const long long tiles = (sims_[s].N + 255) / 256;
        for (long long tI = 0; tI < tiles; ++tI) v.push_back(BlockWork{s, 0, (int)tI});
    }
    Map m;
    m.d = upload(v);
    m.n = (int)v.size();
    return maps_[key] = m;
}

// Staged tiles are laid out back to back in shared memory and filled with 16-byte cp.async copies,
// so every tile size is rounded up to a multiple of four float2 (32 bytes).
static long long round4(long long te) { return (te + 3) & ~3LL; }

void Engine::issue_job(const SpecJob& job, int sim_only) {
    const int comps_in = job.fanout ? 1 : job.nin;
    auto in_launch = [&](int s) { return sim_only < 0 || s == sim_only; };
    auto spec_bytes = [](const SimHost& h) { return (double)h.A * h.B * h.Ch * sizeof(float2); };
    auto open_comps = [&](const SimHost& h, int ncomp) {
        int n = 0;
        for (int c = 0; c < ncomp; ++c) n += host_gate(h, job.gate, c) ? 1 : 0;
        return n;
    };
    // algorithmic bytes of a launch (compulsory HBM reads + writes of its open simulations)
    auto sum_sims = [&](auto in_class, auto per_sim) {
        double b = 0;
        for (int s = 0; s < count(); ++s)
            if (in_launch(s) && in_class(sims_[s]) && t_ < sims_[s].nt) b += per_sim(sims_[s]);
        return b;
    };
    auto classes = [&](auto cls) {
        std::set<int> r;
        for (int s = 0; s < count(); ++s)
            if (in_launch(s)) r.insert(cls(sims_[s]));
        return r;
    };

    // ---- 3D: R2C + forward pass along B per plane, when every simulation of the launch has the
    // same instantiated plane size ----
    int pM = 0, pB = 0;
    bool plane = dim_ == 3 && plane_policy();
    for (int s = 0; plane && s < count(); ++s) {
        if (!in_launch(s)) continue;
        const SimHost& h = sims_[s];
        if (h.C % 2 != 0 || !plane_cluster(h.C / 2, h.B) || (pM && (pM != h.C / 2 || pB != h.B))) plane = false;
        pM = h.C / 2;
        pB = h.B;
    }
    if (plane) {
        RowR2CJob rj{};
        rj.in_field = job.in_field;
        rj.spec_out = job.spec_in;
        rj.gate = job.gate;
        const Map& m = map_planes(comps_in, sim_only);
        const double bytes = sum_sims([](const SimHost&) { return true; },
                                      [&](const SimHost& h) { return open_comps(h, comps_in) * ((double)h.N * 4 + spec_bytes(h)); });
        timed(std::string("plane:") + job.name, bytes, [&] { launch_plane_r2c(st(), d_sims_, d_t_, m.d, m.n, rj, pM, pB); });
    }

    // ---- forward row pass (R2C) ----
    for (int sc : classes(row_class)) {
        if (plane) break;
        if (job.r2c_done && rowr_class(sc) && dim_ >= 2) continue;   // written by the previous job's C2R
        auto in_class = [&](const SimHost& h) { return row_class(h) == sc; };
        long long te = 0;
        for (int s = 0; s < count(); ++s)
            if (in_launch(s) && in_class(sims_[s])) te = std::max(te, (long long)sims_[s].M * (row_lines(sims_[s].M) + 1));
        RowR2CJob rj{};
        rj.in_field = job.in_field;
        rj.spec_out = job.spec_in;
        rj.apply_op = dim_ == 1 ? 1 : 0;
        for (int c = 0; c < kMaxComp; ++c) rj.op[c] = job.op[c];
        rj.gate = job.gate;
        te = round4(te);
        rj.tile_elems = te;
        const bool reg = rowr_class(sc) && !rj.apply_op;
        rj.ahead = reg ? row_ahead(4) : 0;   // 64 registers: four CTAs per SM
        const Map& m = map_rows(reg ? -1 : 0, comps_in, sim_only, sc);
        const double bytes = sum_sims(in_class, [&](const SimHost& h) { return open_comps(h, comps_in) * ((double)h.N * 4 + spec_bytes(h)); });
        const size_t smem = (size_t)(has_fixed_kernel(sc) ? 2 : 3) * te * sizeof(float2);
        if (reg)
            timed(std::string("r2c:") + job.name, bytes, [&] { launch_rowr_r2c(st(), d_sims_, d_t_, m.d, m.n, rj, sc); });
        else
            timed(std::string("r2c:") + job.name, bytes, [&] { launch_row_r2c(st(), d_sims_, d_t_, m.d, m.n, rj, smem, sc); });
    }

    // ---- column passes ----
    // shared memory: two staged tiles (+ staged radial tables and an operator work tile) (+ one
    // ping-pong tile for the runtime plan)
    auto col_launch = [&](int axis, int mode, const char* label, int ncomp_map, auto bytes_of) {
        const bool op = mode == COL_FWD_OP_INV;
        for (int sc : classes([&](const SimHost& h) { return col_class(h, axis); })) {
            auto in_class = [&](const SimHost& h) { return col_class(h, axis) == sc; };
            long long te = 0;
            for (int s = 0; s < count(); ++s)
                if (in_launch(s) && in_class(sims_[s])) {
                    const int n = axis == 0 ? sims_[s].A : sims_[s].B;
                    te = std::max(te, (long long)n * (op ? col_lines_op(n) : col_lines(n)));
                }
            te = round4(te);
            ColJob cj{};
            cj.layout_axis = axis;
            cj.mode = mode;
            cj.spec_in = job.spec_in;
            cj.spec_out = job.spec_out;
            cj.nout = job.nout;
            cj.fanout = job.fanout;
            cj.fanin = mode == COL_FWD_OP_INV ? job.fanin : 0;
            for (int c = 0; c < kMaxComp; ++c) cj.op[c] = job.op[c];
            cj.gate = job.gate;
            cj.tile_elems = te;
            cj.tma_ahead = colp_ahead();
            if (mode == COL_INV) cj.spec_in = job.spec_out, cj.fanout = 0;
            const int pol = map_order_policy();
            const int ord = pol == 2 ? (op ? 3 : 2) : (mode == COL_FWD && pol != 0 ? 1 : 0);
            const Map& m = map_cols(axis, ncomp_map, sim_only, op, sc, 0, ord);
            const double bytes = sum_sims(in_class, bytes_of);
            const long long tiles = sc ? (op ? 4 : 2) : (op ? 5 : 3);
            const size_t smem = (size_t)(tiles * te * sizeof(float2));
            if (op && job.fanin && !(sc && has_colop(sc)))
                throw KwError{KW_ERR_UNSUPPORTED, "fan-in spectral job needs the register column kernel"};
            // register column kernels: the operator pass double-buffered (cola) or one tile per CTA
            // (colop); the in-place passes TMA-fed up to 256 points (colp), double-buffered above
            const int cola = cola_policy();
            if (sc && op && has_colop(sc) && (cola & 1))
                timed(std::string(label) + job.name, bytes, [&] { launch_cola(st(), d_sims_, d_t_, m.d, m.n, cj, sc); });
            else if (sc && op && has_colop(sc)) {
                // the variant the autotuner chose for this pass (kw_tune.cpp), on its own tile map
                const std::string key = colop_key(sc, axis, cj, m.n);
                // the TMA-fed kernel needs every simulation of the launch to have the A-axis maps
                bool tma_ok = dim_ == 3 && axis == 0 && !job.fanin && colop_tma_length(sc);
                for (int s = 0; tma_ok && s < count(); ++s)
                    if (in_launch(s) && in_class(sims_[s])) tma_ok = colp_enabled(sims_[s], 0) && sims_[s].dev.tmaps;
                if (tune_mode_) {
                    tune_colop(sc, axis, ncomp_map, sim_only, cj, key, tma_ok);
                } else {
                    const ColopVariant v = colop_choice(sc, key, tma_ok);
                    const Map& mv = map_cols(axis, ncomp_map, sim_only, op, sc, colop_tile(sc, v.r1), ord);
                    timed(std::string(label) + job.name, bytes,
                          [&] { launch_colop(st(), d_sims_, d_t_, mv.d, mv.n, cj, sc, v, d_flag_ + 1); });
                }
            }
            else if (sc && !op && has_colp(sc) && !(cola & 2))
                timed(std::string(label) + job.name, bytes,
                      [&] { launch_colp(st(), d_sims_, d_t_, m.d, m.n, cj, sc, d_flag_ + 1); });
            else if (sc && !op && has_colop(sc) && !(cola & 4))
                timed(std::string(label) + job.name, bytes, [&] { launch_cola(st(), d_sims_, d_t_, m.d, m.n, cj, sc); });
            else
                timed(std::string(label) + job.name, bytes, [&] { launch_col(st(), d_sims_, d_t_, m.d, m.n, cj, smem, sc); });
        }
    };
    int spec_final = job.spec_in;
    if (dim_ >= 2) {
        if (dim_ == 3 && !plane)
            col_launch(1, COL_FWD, "colB_fwd:", comps_in,
                       [&](const SimHost& h) { return open_comps(h, comps_in) * 2 * spec_bytes(h); });
        const int last = dim_ == 3 ? 0 : 1;
        col_launch(last, COL_FWD_OP_INV, last == 0 ? "colA_op:" : "colB_op:", job.fanout ? 1 : job.nout,
                   [&](const SimHost& h) {
                       const int no = open_comps(h, job.fanout ? 1 : job.nout);
                       if (no == 0) return 0.0;
                       const double tables = job.op[0].radial != RT_NONE ? (double)h.A * h.B * h.Ch * 4 : 0.0;
                       if (job.fanin) return spec_bytes(h) * (job.fanin + 1) + tables * job.fanin;
                       return job.fanout ? spec_bytes(h) * (1 + job.nout) + tables : no * (2 * spec_bytes(h) + tables);
                   });
        spec_final = job.spec_out;
        if (dim_ == 3)
            col_launch(1, COL_INV, "colB_inv:", job.nout, [&](const SimHost& h) {
                return (job.fanout ? (open_comps(h, 1) ? job.nout : 0) : open_comps(h, job.nout)) * 2 * spec_bytes(h);
            });
    }

    // ---- inverse row pass (C2R) + epilogue ----
    const int ncta = job.coupled ? job.nout : 1;
    for (int sc : classes(row_class)) {
        auto in_class = [&](const SimHost& h) { return row_class(h) == sc; };
        long long te = 0, aux_floats = 0;
        for (int s = 0; s < count(); ++s)
            if (in_launch(s) && in_class(sims_[s])) {
                const SimHost& h = sims_[s];
                te = std::max(te, (long long)(h.C % 2 ? h.M : h.M + 1) * (c2r_lines(h.M) + 1));
                const int rpc = std::max(1, c2r_lines(h.M) / ncta);
                aux_floats = std::max(aux_floats, (long long)aux_slots(h, job.epi) * rpc * h.C);
            }
        te = round4(te);
        aux_floats = (aux_floats + 3) & ~3LL;
        RowC2RJob cj{};
        cj.spec_in = spec_final;
        cj.ncomp = ncta;
        cj.epi = job.epi;
        cj.out_field = job.out_field;
        cj.gate = job.gate;
        cj.generic = has_fixed_kernel(sc) ? 0 : 1;
        cj.tape = job.tape;
        cj.tile_elems = te;
        const bool reg = rowr_class(sc);
        cj.prefetch = c2r_prefetch() ? 1 : 0;
        cj.ahead = reg && ncta == 1 ? row_ahead(3) : 0;   // three CTAs per SM (the 128-point epilogues)
        cj.fwd = job.fwd_spec >= 0 && reg && dim_ >= 2;
        cj.fwd_spec = job.fwd_spec;
        const Map& m = map_rows(reg ? -2 : ncta, job.coupled ? 1 : job.nout, sim_only, sc, alternate_order());
        const double bytes = sum_sims(in_class, [&](const SimHost& h) {
            int no = job.coupled ? (open_comps(h, 1) ? job.nout : 0) : open_comps(h, job.nout);
            if (job.epi == EPI_EOS_ABS && no) no = h.dev.absorb == 3 ? 2 : 1;
            if (no == 0) return 0.0;
            double b = no * spec_bytes(h) + (double)h.N * epi_bytes(h, job.epi, job.coupled ? 1 : no);
            if (cj.fwd) {   // the fused R2C's spectra; the density epilogue then keeps rho0 div u on chip
                if (job.epi == EPI_VEL || job.epi == EPI_ADJ_VEL || job.epi == EPI_ADJ_VEL_RHO) b += no * spec_bytes(h);
                else if (h.dev.absorb >= 2) b += (h.dev.absorb == 3 ? 2 : 1) * spec_bytes(h) - (double)h.N * 4;
            }
            return b;
        });
        const size_t smem = (size_t)(has_fixed_kernel(sc) ? 2 : 3) * te * sizeof(float2) + (size_t)aux_floats * sizeof(float);
        if (reg)
            timed(std::string("c2r:") + job.name, bytes, [&] { launch_rowr_c2r(st(), d_sims_, d_t_, m.d, m.n, cj, sc); });
        else
            timed(std::string("c2r:") + job.name, bytes, [&] { launch_row_c2r(st(), d_sims_, d_t_, m.d, m.n, cj, smem, sc); });
    }
}

}  // namespace kw
