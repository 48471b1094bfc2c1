// kw_tune.cpp — the autotuner of the operator column pass (kw_pass_colop.cu).
//
// The operator pass of a spectral job (forward transform, k-space operator, inverse transform(s)
// along the last layout axis) comes in variants per line length: values per thread R1 (so lines
// per CTA) and a launch bound of resident CTAs per SM. Which is fastest depends on the length, the
// number of outputs, the tile count and the GPU. At the end of kw_sim_create / kw_batch_create the
// engine issues one time step in tune mode: every launch is skipped except the operator passes,
// whose variants are each timed with CUDA events (two warm-up launches, then ten) on the job's own
// tile map, and the fastest is kept for that key. The spectra the passes overwrite are scratch
// between jobs, so timing them before the first step changes no result.
//
// Keys: "colop/<length>/<layout axis>/<outputs>/<fan-out>/<log2 tiles>". Where the launch allows
// it (3D, along A, lengths 128 and 256, tensor maps present) the TMA-fed warp-specialised kernel is
// a further candidate (minb = kColopTma). Choices are cached in
// memory for the process and in a JSON file per GPU model: $KW_TUNE_CACHE if set, else
// $HOME/.cache/kwave_b200/tune_<gpu>.json. KW_AUTOTUNE=0 turns tuning off (every pass takes its
// default variant); KW_COLOP_VARIANT=r1,minb forces that variant wherever the length has it.
//
// Variants with the same R1 run the same arithmetic in the same order, so they give bit-identical
// results; a different R1 splits the transform into different radix stages and its results differ
// in the last bits (relative L2 ~1e-7).
#include "kw_engine.h"

#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <sys/stat.h>
#include <unistd.h>

namespace kw {

namespace {

struct TuneEntry {
    ColopVariant v;
    double us;
};

class TuneCache {
public:
    static TuneCache& get() {
        static TuneCache c;
        return c;
    }
    bool find(const std::string& key, ColopVariant* v) {
        std::lock_guard<std::mutex> lock(mu_);
        load_locked();
        auto it = map_.find(key);
        if (it == map_.end()) return false;
        *v = it->second.v;
        return true;
    }
    void put(const std::string& key, ColopVariant v, double us) {
        std::lock_guard<std::mutex> lock(mu_);
        load_locked();
        map_[key] = TuneEntry{v, us};
        save_locked();
    }

private:
    std::mutex mu_;
    std::map<std::string, TuneEntry> map_;
    bool loaded_ = false;
    std::string path_;

    static std::string gpu_tag() {
        int dev = 0;
        cudaDeviceProp p{};
        if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&p, dev) != cudaSuccess) {
            cudaGetLastError();
            return "gpu";
        }
        std::string s;
        for (const char* c = p.name; *c; ++c) s += std::isalnum((unsigned char)*c) ? *c : '_';
        return s;
    }
    // $KW_TUNE_CACHE (read on every lookup: tests change it), else the per-GPU default, resolved
    // once per process (it queries the device properties and creates the directory)
    std::string resolve_path() {
        if (const char* e = std::getenv("KW_TUNE_CACHE")) return e;
        if (!default_resolved_) {
            default_resolved_ = true;
            if (const char* h = std::getenv("HOME")) {
                const std::string dir = std::string(h) + "/.cache/kwave_b200";
                mkdir((std::string(h) + "/.cache").c_str(), 0755);
                mkdir(dir.c_str(), 0755);
                default_path_ = dir + "/tune_" + gpu_tag() + ".json";
            }
        }
        return default_path_;
    }
    bool default_resolved_ = false;
    std::string default_path_;
    std::string gpu_name_;
    // (re)load when the cache file in effect changed (KW_TUNE_CACHE set or changed in the process)
    void load_locked() {
        const std::string want = resolve_path();
        if (loaded_ && want == path_) return;
        loaded_ = true;
        map_.clear();
        path_ = want;
        if (path_.empty()) return;
        std::ifstream f(path_);
        std::string line;
        while (std::getline(f, line)) {
            // "key": {"r1": R, "minb": M, "us": T}
            const size_t q0 = line.find('"'), q1 = q0 == std::string::npos ? q0 : line.find('"', q0 + 1);
            if (q1 == std::string::npos || line.compare(q0 + 1, 6, "colop/") != 0) continue;
            TuneEntry e{};
            if (std::sscanf(line.c_str() + q1 + 1, ": {\"r1\": %d, \"minb\": %d, \"us\": %lf", &e.v.r1, &e.v.minb, &e.us) == 3)
                map_[line.substr(q0 + 1, q1 - q0 - 1)] = e;
        }
    }
    void save_locked() {
        if (path_.empty()) return;
        std::ostringstream o;
        if (gpu_name_.empty()) gpu_name_ = gpu_tag();
        o << "{\n \"kernel\": \"k_colop\",\n \"gpu\": \"" << gpu_name_ << "\",\n \"choices\": {\n";
        size_t i = 0;
        for (const auto& kv : map_) {
            char buf[96];
            std::snprintf(buf, sizeof buf, "{\"r1\": %d, \"minb\": %d, \"us\": %.3f}", kv.second.v.r1, kv.second.v.minb,
                          kv.second.us);
            o << "  \"" << kv.first << "\": " << buf << (++i < map_.size() ? "," : "") << "\n";
        }
        o << " }\n}\n";
        const std::string tmp = path_ + ".tmp" + std::to_string((long)getpid());
        {
            std::ofstream f(tmp);
            if (!f) return;
            f << o.str();
        }
        std::rename(tmp.c_str(), path_.c_str());   // whole-file replace: concurrent writers never interleave
    }
};

// launches per candidate: untimed, then timed back to back (the mean is kept)
constexpr int kTuneWarm = 2, kTuneReps = 10;

bool autotune_enabled() {
    const char* e = std::getenv("KW_AUTOTUNE");
    return !(e && e[0] == '0');
}

// the variants of length n for this launch: the register ones, and the TMA-fed one where the
// launch can take it (KW_COLOP_TMA=0 leaves it out)
int candidates(int n, bool tma_ok, ColopVariant* out) {
    int nc = colop_variants(n, out, 15);
    const char* e = std::getenv("KW_COLOP_TMA");
    if (tma_ok && colop_tma_length(n) && !(e && e[0] == '0')) out[nc++] = ColopVariant{16, kColopTma};
    return nc;
}

bool forced_variant(int n, bool tma_ok, ColopVariant* v) {
    const char* e = std::getenv("KW_COLOP_VARIANT");
    if (!e) return false;
    ColopVariant f{};
    if (std::sscanf(e, "%d,%d", &f.r1, &f.minb) != 2) return false;
    ColopVariant cands[16];
    const int nc = candidates(n, tma_ok, cands);
    for (int k = 0; k < nc; ++k)
        if (cands[k].r1 == f.r1 && cands[k].minb == f.minb) {
            *v = f;
            return true;
        }
    return false;
}

}  // namespace

std::string Engine::colop_key(int n, int axis, const ColJob& cj, int ntiles) const {
    const int nouts = cj.fanout ? cj.nout : 1;
    int lg = 0;
    while ((1 << (lg + 1)) <= std::max(ntiles, 1)) ++lg;
    return "colop/" + std::to_string(n) + "/" + std::to_string(axis) + "/" + std::to_string(nouts) + "/" +
           std::to_string(cj.fanout) + "/" + std::to_string(lg);
}

ColopVariant Engine::colop_choice(int n, const std::string& key, bool tma_ok) const {
    ColopVariant cands[16];
    const int nc = candidates(n, tma_ok, cands);
    ColopVariant v = cands[0];
    if (forced_variant(n, tma_ok, &v)) return v;
    ColopVariant c;
    if (autotune_enabled() && TuneCache::get().find(key, &c))
        for (int k = 0; k < nc; ++k)
            if (cands[k].r1 == c.r1 && cands[k].minb == c.minb) v = c;   // only a choice valid here
    return v;
}

// Time every variant of the operator pass on its own tile map and keep the fastest (tune mode).
void Engine::tune_colop(int n, int axis, int ncomp_map, int sim_only, const ColJob& cj, const std::string& key,
                        bool tma_ok) {
    ColopVariant cur;
    if (!autotune_enabled() || TuneCache::get().find(key, &cur)) return;
    ColopVariant cands[16];
    const int nc = candidates(n, tma_ok, cands);
    if (nc <= 1) {
        TuneCache::get().put(key, cands[0], 0.0);
        return;
    }
    cudaEvent_t a, b;
    check(cudaEventCreate(&a), "event");
    check(cudaEventCreate(&b), "event");
    int best = 0;
    double best_us = 1e300;
    for (int k = 0; k < nc; ++k) {
        const Map& m = map_cols(axis, ncomp_map, sim_only, true, n, colop_tile(n, cands[k].r1));
        for (int r = 0; r < kTuneWarm; ++r) launch_colop(st(), d_sims_, d_t_, m.d, m.n, cj, n, cands[k], d_flag_ + 1);
        check(cudaEventRecord(a, st()), "event");
        for (int r = 0; r < kTuneReps; ++r) launch_colop(st(), d_sims_, d_t_, m.d, m.n, cj, n, cands[k], d_flag_ + 1);
        check(cudaEventRecord(b, st()), "event");
        check(cudaEventSynchronize(b), "tune sync");
        check(cudaGetLastError(), "tune launch");
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        const double us = 1e3 * ms / kTuneReps;
        if (us < best_us) {
            best_us = us;
            best = k;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    TuneCache::get().put(key, cands[best], best_us);
}

// One time step in tune mode (see the top of this file); the state is reset afterwards.
void Engine::autotune() {
    if (!autotune_enabled() || as_mode_) return;
    tune_mode_ = true;
    try {
        issue_step(false);
    } catch (...) {
        tune_mode_ = false;
        throw;
    }
    tune_mode_ = false;
    check(cudaStreamSynchronize(st()), "tune sync");
    reset();
}

}  // namespace kw
