// kw_engine.h — host engine: setup (FP64 precompute), step sequencing, recording, outputs.
#pragma once

#include <chrono>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/kwave_cuda.h"
#include "kw_common.h"
#include "kw_async.cuh"
#include "kw_kernels.cuh"

namespace kw {

struct Context {
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    std::string err;
    int fail(int code, const std::string& msg) { err = msg; return code; }

    // Device blocks of destroyed simulations, kept for the next create on this context (keyed by
    // their rounded size; a create of the same problem finds every block it needs), up to a
    // quarter of the device's memory. A failed cudaMalloc releases the cache and tries once more.
    // kw_context_destroy frees it.
    std::mutex cache_mu;
    std::multimap<size_t, void*> cache;
    size_t cached_bytes = 0;
    size_t cache_cap = 0;   // at most this much is kept (a quarter of device memory)
    static size_t round_block(size_t bytes) {
        return bytes >= (1u << 20) ? (bytes + (2u << 20) - 1) & ~(size_t)((2u << 20) - 1) : (bytes + 511) & ~(size_t)511;
    }
    void* cache_take(size_t rounded);
    void cache_put(void* p, size_t rounded);
    void cache_release();

    // Two pinned staging buffers for host -> device uploads of large inputs: the host copy of one
    // chunk (on several threads) overlaps the DMA of the previous one
    static constexpr size_t kStageBytes = 8u << 20;
    std::mutex stage_mu;
    void* stage[2] = {nullptr, nullptr};
    cudaEvent_t stage_ev[2] = {nullptr, nullptr};
    bool stage_failed = false;   // no pinned memory could be had: plain copies

    ~Context();
};

// A status-carrying error used inside the engine; converted to kw_status at the ABI.
struct KwError {
    int code;
    std::string msg;
};

// Device address of the allocation-free scratch array on `device` (kw_noalloc.cu).
void* noalloc_scratch(int device);

struct SimHost;
// true when the column pass along `layout_axis` (0 = A, 1 = B) of this simulation runs the
// TMA-fed warp-specialised kernel (kw_tmaps.cpp)
bool colp_enabled(const SimHost& h, int layout_axis);

// Host-side record of one simulation.
struct SimHost {
    kw_sim_desc d{};               // scalar fields of the descriptor (pointers not retained)
    int dim = 0, A = 1, B = 1, C = 1, Ch = 1, Cp = 2;
    int M = 1;                     // complex length of the row transform (C/2, or C when C is odd)
    int n_ref[3] = {1, 1, 1};      // nx, ny, nz
    double d_ref[3] = {1, 1, 1};
    long long N = 0, Ns = 0;
    int nt = 0;
    double cref = 0;
    bool record_p = false, record_u = false, record_ufinal = false;
    bool p_series = false, u_series = false, p_agg = false, u_agg = false;
    int npts = 0;
    bool psrc_precorrect = false;  // single-row additive p source: corrected once at setup
    float* p0s = nullptr;          // smoothed initial pressure (device) or null
    SimDev dev{};
};

class Engine {
public:
    explicit Engine(Context* ctx);
    ~Engine();
    void create(const kw_sim_desc* descs, int count);
    void reset();
    void step(int nsteps);
    void run(const kw_callbacks* cb);
    int synchronize();             // returns KW_OK or KW_ERR_NONFINITE
    int t() const { return t_; }
    int count() const { return (int)sims_.size(); }
    const SimHost& sim(int i) const { return sims_[i]; }
    size_t output_size(int i, int field) const;
    void get_output(int i, int field, float* dst, size_t count);
    const float* device_field(int i, int field, size_t* count) const;
    struct KernelTiming {
        std::string name;
        double ms;
        double bytes;
    };
    // Run `reps` time steps launch by launch with CUDA events around each launch; returns the mean
    // device time and the algorithmic HBM bytes of every launch of one step, in launch order.
    std::vector<KernelTiming> profile_step(int reps);
    // Standalone staggered spectral derivative of a device field (kw_derivative.cpp).
    void create_derivative(int dim, const int* n, const double* d, int axis, int shift, const float* in, float* out);
    void run_derivative();
    // Discrete adjoint of a single simulation's misfit (kw_adjoint.cpp).
    void adjoint(const kw_sim_desc& d, kw_adjoint_desc& a);
    // Take every device buffer from [base, base + bytes) instead of cudaMalloc (call before create).
    void set_arena(void* base, size_t bytes) {
        arena_ = static_cast<char*>(base);
        arena_size_ = bytes;
        arena_used_ = 0;
    }

private:
    struct Map {
        BlockWork* d = nullptr;
        int n = 0;
    };
    struct SpecJob {
        int in_field = FS_P;
        int nin = 1;
        int fanout = 0;
        int nout = 1;
        OpSpec op[kMaxComp]{};
        int spec_in = 0, spec_out = 0;
        int epi = EPI_STORE;
        int out_field = FS_TMP;
        int coupled = 0;
        int gate = GATE_NONE;
        int comp_mask = 7;        // which components take part (per-comp jobs)
        int fanin = 0;            // the operator pass sums the nin inputs into output 0 (register column kernel)
        int tape = 0;             // the epilogue also stores the adjoint tape of the step
        int fwd_spec = -1;        // >= 0: the C2R also writes the next job's input spectra (row fusion)
        int r2c_done = 0;         // the previous job's C2R wrote this job's input spectra (register rows)
        const char* name = "job";
    };
    struct ProfRec {
        std::string name;
        double bytes;
        cudaEvent_t a, b;
    };
    template <class F>
    void timed(const std::string& name, double bytes, F&& f) {
        if (tune_mode_ || dry_) return;   // only the operator passes run (and are timed) in tune mode
        if (!prof_) { f(); return; }
        ProfRec r{name, bytes, nullptr, nullptr};
        cudaEventCreate(&r.a);
        cudaEventCreate(&r.b);
        cudaEventRecord(r.a, st());
        f();
        cudaEventRecord(r.b, st());
        prof_->push_back(r);
    }
    bool host_gate(const SimHost& h, int gate, int comp) const;
    double epi_bytes(const SimHost& h, int epi, int ncomp) const;
    int aux_slots(const SimHost& h, int epi) const;

    void* dalloc(size_t bytes);
    template <class T>
    T* upload(const std::vector<T>& v) {
        if (v.empty()) return nullptr;
        T* p = (T*)dalloc(v.size() * sizeof(T));
        check(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st()), "upload");
        return p;
    }
    // device copy of n host floats
    float* upload_floats(const float* src, long long n) {
        float* p = (float*)dalloc((size_t)n * sizeof(float));
        upload_host(p, src, (size_t)n * sizeof(float));
        return p;
    }
    // host -> device copy of a caller's (pageable) buffer, staged through the context's pinned
    // buffers when it is large
    void upload_host(void* dst, const void* src, size_t bytes);
    void download_host(void* dst, const void* src, size_t bytes);   // synchronous, staged when large
    bool stage_ready_locked();   // with Context::stage_mu held
    void check(cudaError_t e, const char* what);
    cudaStream_t st() const { return st_override_ ? st_override_ : ctx_->stream; }

    void setup_sim(int s, const kw_sim_desc& d);
    void build_tensor_maps(SimHost& h, SimDev& v);   // kw_tmaps.cpp
    void check_kernel_error();
    void build_plan(FFTPlanDev& pl, int n);
    void smooth_field(int s, float* field);
    const Map& map_rows(int lines_per_row, int ncomp, int sim_only, int sclass, bool reverse = false);
    // tw > 0: tiles of tw columns (the register operator pass of the chosen variant)
    // order: 0 forwards, 1 backwards, 2 / 3 column-chunk-major forwards / backwards (kw_jobs.cpp)
    const Map& map_cols(int axis, int ncomp, int sim_only, bool op, int sclass, int tw = 0, int order = 0);
    const Map& map_elems(int sim_only);
    const Map& map_planes(int ncomp, int sim_only);
    void issue_job(const SpecJob& job, int sim_only);
    bool fuse_rows() const;   // row fusion of consecutive jobs allowed (not with the plane pass; KW_FUSE_ROWS=0 off)
    void issue_step(bool first);
    int capture_graph();   // returns the variant captured / in use for the current step
    void finalize_outputs();

    Context* ctx_;
    std::vector<SimHost> sims_;
    std::vector<std::pair<void*, size_t>> allocs_;   // device blocks and their rounded sizes
    SimDev* d_sims_ = nullptr;
    int* d_t_ = nullptr;
    unsigned int* d_tickc_ = nullptr;   // see launch_sample
    int* d_flag_ = nullptr;
    const float** d_p0s_ = nullptr;
    unsigned int* d_red_ = nullptr;
    int t_ = 0;
    int dim_ = 0;
    int max_psrc_ = 0, max_usrc_ = 0, max_pts_ = 0, max_dir_ = 0;
    bool any_p_direct_ = false, any_p_add_ = false, any_u_direct_ = false, any_u_add_ = false;
    bool any_abs_ = false, any_p0_ = false, any_recu_ = false, any_recp_ = false;
    int max_A_ = 1, max_B_ = 1, max_M_ = 1;
    std::map<std::tuple<int, int, int, int, int>, Map> maps_;
    // the steady step as CUDA graphs: [1] while a precorrected pressure source of some simulation
    // is still injecting (the density epilogue adds it), [0] otherwise
    cudaGraph_t graph_[2] = {nullptr, nullptr};
    cudaGraphExec_t graph_exec_[2] = {nullptr, nullptr};
    cudaStream_t graph_stream_[2] = {nullptr, nullptr};
    bool psrc_live() const;
    std::vector<ProfRec>* prof_ = nullptr;
    int deriv_axis_ = 0, deriv_shift_ = 1;
    char* arena_ = nullptr;
    size_t arena_size_ = 0, arena_used_ = 0;
    bool finalized_ = false;
    bool tape_mode_ = false;   // adjoint: steps are captured with the tape epilogues
    // single-row additive pressure sources may be precorrected at setup (SimDev::psrc_q); the
    // adjoint and the axisymmetric solver keep the per-step correction job
    bool precorrect_ok_ = true;
    void precorrect_psrc(int s);
    // autotuner of the operator column pass (kw_tune.cpp)
    bool tune_mode_ = false;
    bool dry_ = false;
    bool trace_ = false;   // KW_TRACE_SETUP=1
    std::chrono::steady_clock::time_point trace_last_;
    void trace_phase(const char* what);   // issue_step creates the tile maps but launches nothing (before a graph capture)
    std::string colop_key(int n, int axis, const ColJob& cj, int ntiles) const;
    ColopVariant colop_choice(int n, const std::string& key, bool tma_ok) const;
    void tune_colop(int n, int axis, int ncomp_map, int sim_only, const ColJob& cj, const std::string& key,
                    bool tma_ok);
    void autotune();
    cudaStream_t st_override_ = nullptr;   // adjoint: the reverse sweep's own stream while it issues work
    // axisymmetric solver (kw_axisym.cpp): sims_[0] is the [nx][ny] simulation, car_ / d_car_ the
    // descriptor of its 4x radial expansion that the spectral jobs run on
    bool as_mode_ = false;
    SimHost car_;
    SimDev* d_car_ = nullptr;
    void create_as_carrier();
    void issue_step_as(bool first);
    int finalized_t_ = -1;
    static constexpr int kFinitePoll = 64;   // steps between the non-finite checks of run()
    int* poll_host_ = nullptr;                // pinned copy of the non-finite flag
    cudaEvent_t poll_ev_ = nullptr;
    long long wait_cycles_ = kWaitCycles;     // SimDev::wait_cycles (test hook KW_TEST_STALL_COLUMN_PASS)
    int test_stall_ = 0;                      // SimDev::test_stall (same hook)
    int fail_alloc_ = 0, nalloc_ = 0;         // test hook KW_TEST_FAIL_ALLOC
    // finalised aggregate outputs per sim (device)
    struct Outs {
        float* iavg[kMaxComp] = {nullptr, nullptr, nullptr};
    };
    std::vector<Outs> outs_;
};

}  // namespace kw
