// kw_capi.cpp — the extern "C" boundary declared in include/kwave_cuda.h.
//
// Every entry point catches engine errors and returns a kw_status; nothing aborts the process.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "../../include/kwave_cuda.h"
#include "kw_engine.h"

struct kw_context {
    kw::Context c;
};
struct kw_sim {
    kw_context* ctx;
    kw::Engine* eng;
};
struct kw_batch {
    kw_context* ctx;
    kw::Engine* eng;
};

static thread_local std::string g_last_global;

template <class F>
static int guarded(kw_context* ctx, F&& f) {
    try {
        if (ctx) cudaSetDevice(ctx->c.device);
        return f();
    } catch (const kw::KwError& e) {
        if (ctx) ctx->c.err = e.msg;
        g_last_global = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        if (ctx) ctx->c.err = "host allocation failed";
        return KW_ERR_OOM;
    } catch (...) {
        if (ctx) ctx->c.err = "unexpected error";
        return KW_ERR_CUDA;
    }
}

extern "C" {

const char* kw_version(void) { return "kwave-b200 0.1.0 (sm_100a)"; }
int kw_abi_version(void) { return KW_ABI_VERSION; }

void kw_sim_desc_init(kw_sim_desc* d) {
    if (!d) return;
    std::memset(d, 0, sizeof(*d));
    d->abi_version = KW_ABI_VERSION;
    d->dim = 2;
    d->nx = d->ny = d->nz = 1;
    d->dx = d->dy = d->dz = 1.0;
    d->pml_size = 20;
    d->pml_alpha = 2.0;
    d->smooth_p0 = 1;
    d->c_ref = NAN;
    d->alpha_power = NAN;
    d->alpha_mode = KW_ABSORPTION_NONE;
    d->p_mode = KW_SOURCE_ADDITIVE;
    d->u_mode = KW_SOURCE_ADDITIVE;
    d->record = KW_RECORD_P;
    d->directivity_size = NAN;
    d->directivity_pattern = KW_DIRECTIVITY_PRESSURE;
}

int kw_context_create(int device, kw_context** out) {
    if (!out) return KW_ERR_INVALID;
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        g_last_global = std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "count is 0");
        return KW_ERR_CUDA;
    }
    if (device < 0 || device >= n) { g_last_global = "device index out of range"; return KW_ERR_INVALID; }
    auto* ctx = new (std::nothrow) kw_context();
    if (!ctx) return KW_ERR_OOM;
    ctx->c.device = device;
    int st = guarded(ctx, [&]() {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) throw kw::KwError{KW_ERR_CUDA, "cudaGetDeviceProperties failed"};
        if (prop.major < 10) throw kw::KwError{KW_ERR_UNSUPPORTED, std::string("this library is built for sm_100a; device is ") + prop.name};
        if (cudaStreamCreateWithFlags(&ctx->c.own, cudaStreamNonBlocking) != cudaSuccess)
            throw kw::KwError{KW_ERR_CUDA, "stream creation failed"};
        ctx->c.stream = ctx->c.own;
        kw::init_kernel_attributes();
        return KW_OK;
    });
    if (st != KW_OK) { delete ctx; return st; }
    *out = ctx;
    return KW_OK;
}

int kw_context_set_stream(kw_context* ctx, void* stream) {
    if (!ctx) return KW_ERR_INVALID;
    ctx->c.stream = stream ? (cudaStream_t)stream : ctx->c.own;
    return KW_OK;
}

void kw_context_destroy(kw_context* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->c.device);
    if (ctx->c.own) cudaStreamDestroy(ctx->c.own);
    delete ctx;
}

const char* kw_last_error_message(const kw_context* ctx) {
    return ctx ? ctx->c.err.c_str() : g_last_global.c_str();
}

int kw_sim_create(kw_context* ctx, const kw_sim_desc* desc, kw_sim** out) {
    if (!ctx || !desc || !out) return KW_ERR_INVALID;
    *out = nullptr;
    auto* eng = new (std::nothrow) kw::Engine(&ctx->c);
    if (!eng) return KW_ERR_OOM;
    int st = guarded(ctx, [&]() { eng->create(desc, 1); return KW_OK; });
    if (st != KW_OK) { delete eng; return st; }
    *out = new kw_sim{ctx, eng};
    return KW_OK;
}

int kw_sim_run(kw_sim* sim, const kw_callbacks* cb) {
    if (!sim) return KW_ERR_INVALID;
    return guarded(sim->ctx, [&]() { sim->eng->run(cb); return sim->eng->synchronize(); });
}

int kw_sim_reset(kw_sim* sim) {
    if (!sim) return KW_ERR_INVALID;
    return guarded(sim->ctx, [&]() { sim->eng->reset(); return KW_OK; });
}

int kw_sim_step(kw_sim* sim, int nsteps) {
    if (!sim || nsteps < 0) return KW_ERR_INVALID;
    return guarded(sim->ctx, [&]() { sim->eng->step(nsteps); return KW_OK; });
}

int kw_sim_synchronize(kw_sim* sim) {
    if (!sim) return KW_ERR_INVALID;
    return guarded(sim->ctx, [&]() { return sim->eng->synchronize(); });
}

int kw_sim_current_step(const kw_sim* sim, int* t) {
    if (!sim || !t) return KW_ERR_INVALID;
    *t = sim->eng->t();
    return KW_OK;
}

int kw_sim_num_sensor_points(const kw_sim* sim, int* count) {
    if (!sim || !count) return KW_ERR_INVALID;
    *count = sim->eng->sim(0).npts;
    return KW_OK;
}

int kw_sim_output_size(const kw_sim* sim, int field, size_t* count) {
    if (!sim || !count || field < 0 || field >= KW_FIELD_COUNT) return KW_ERR_INVALID;
    *count = sim->eng->output_size(0, field);
    return KW_OK;
}

int kw_sim_get_output(kw_sim* sim, int field, float* dst, size_t count) {
    if (!sim || !dst || field < 0 || field >= KW_FIELD_COUNT) return KW_ERR_INVALID;
    return guarded(sim->ctx, [&]() { sim->eng->get_output(0, field, dst, count); return KW_OK; });
}

int kw_sim_device_field(kw_sim* sim, int field, const float** dptr, size_t* count) {
    if (!sim || !dptr || !count) return KW_ERR_INVALID;
    *dptr = sim->eng->device_field(0, field, count);
    return *dptr ? KW_OK : KW_ERR_INVALID;
}

int kw_sim_profile_step(kw_sim* sim, int reps, kw_kernel_timing* out, int max_entries, int* n_entries) {
    if (!sim || !out || !n_entries || reps <= 0) return KW_ERR_INVALID;
    return guarded(sim->ctx, [&]() {
        auto v = sim->eng->profile_step(reps);
        const int n = std::min<int>((int)v.size(), max_entries);
        for (int i = 0; i < n; ++i) {
            std::memset(out[i].name, 0, sizeof(out[i].name));
            std::strncpy(out[i].name, v[i].name.c_str(), sizeof(out[i].name) - 1);
            out[i].ms = v[i].ms;
            out[i].bytes = v[i].bytes;
        }
        *n_entries = n;
        return KW_OK;
    });
}

void kw_sim_destroy(kw_sim* sim) {
    if (!sim) return;
    cudaSetDevice(sim->ctx->c.device);
    delete sim->eng;
    delete sim;
}

int kw_spectral_derivative(kw_context* ctx, int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                           int axis, int shift, const float* d_in, float* d_out) {
    if (!ctx) return KW_ERR_INVALID;
    return guarded(ctx, [&]() {
        const int n[3] = {nx, ny, nz};
        const double d[3] = {dx, dy, dz};
        kw::Engine eng(&ctx->c);
        eng.create_derivative(dim, n, d, axis, shift, d_in, d_out);
        eng.run_derivative();
        return KW_OK;
    });
}

int kw_spectral_derivative_noalloc(kw_context* ctx, int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                                   int axis, int shift, const float* d_in, float* d_out) {
    if (!ctx) return KW_ERR_INVALID;
    return guarded(ctx, [&]() {
        const int n[3] = {nx, ny, nz};
        const double d[3] = {dx, dy, dz};
        kw::Engine eng(&ctx->c);
        eng.set_arena(kw::noalloc_scratch(ctx->c.device), KW_NOALLOC_SCRATCH_BYTES);
        eng.create_derivative(dim, n, d, axis, shift, d_in, d_out);
        eng.run_derivative();
        return KW_OK;
    });
}

void kw_adjoint_desc_init(kw_adjoint_desc* a) {
    if (!a) return;
    std::memset(a, 0, sizeof(*a));
    a->abi_version = KW_ABI_VERSION;
    a->policy = KW_CHECKPOINT_SQRT;
}

int kw_adjoint_run(kw_context* ctx, const kw_sim_desc* desc, kw_adjoint_desc* adj) {
    if (!ctx || !desc || !adj) return KW_ERR_INVALID;
    return guarded(ctx, [&]() {
        kw::Engine eng(&ctx->c);
        eng.adjoint(*desc, *adj);
        return KW_OK;
    });
}

int kw_batch_create(kw_context* ctx, const kw_sim_desc* descs, int count, kw_batch** out) {
    if (!ctx || !descs || count <= 0 || !out) return KW_ERR_INVALID;
    *out = nullptr;
    auto* eng = new (std::nothrow) kw::Engine(&ctx->c);
    if (!eng) return KW_ERR_OOM;
    int st = guarded(ctx, [&]() { eng->create(descs, count); return KW_OK; });
    if (st != KW_OK) { delete eng; return st; }
    *out = new kw_batch{ctx, eng};
    return KW_OK;
}

int kw_batch_run(kw_batch* b, const kw_callbacks* cb) {
    if (!b) return KW_ERR_INVALID;
    return guarded(b->ctx, [&]() { b->eng->run(cb); return b->eng->synchronize(); });
}

int kw_batch_reset(kw_batch* b) {
    if (!b) return KW_ERR_INVALID;
    return guarded(b->ctx, [&]() { b->eng->reset(); return KW_OK; });
}

int kw_batch_step(kw_batch* b, int nsteps) {
    if (!b || nsteps < 0) return KW_ERR_INVALID;
    return guarded(b->ctx, [&]() { b->eng->step(nsteps); return KW_OK; });
}

int kw_batch_synchronize(kw_batch* b) {
    if (!b) return KW_ERR_INVALID;
    return guarded(b->ctx, [&]() { return b->eng->synchronize(); });
}

int kw_batch_output_size(const kw_batch* b, int index, int field, size_t* count) {
    if (!b || !count || field < 0 || field >= KW_FIELD_COUNT || index < 0 || index >= b->eng->count()) return KW_ERR_INVALID;
    *count = b->eng->output_size(index, field);
    return KW_OK;
}

int kw_batch_get_output(kw_batch* b, int index, int field, float* dst, size_t count) {
    if (!b || !dst || field < 0 || field >= KW_FIELD_COUNT || index < 0 || index >= b->eng->count()) return KW_ERR_INVALID;
    return guarded(b->ctx, [&]() { b->eng->get_output(index, field, dst, count); return KW_OK; });
}

void kw_batch_destroy(kw_batch* b) {
    if (!b) return;
    cudaSetDevice(b->ctx->c.device);
    delete b->eng;
    delete b;
}

}  // extern "C"
