/*
 * kwave_cuda.h — C ABI of the B200 (sm_100a) k-space pseudospectral fluid solver.
 *
 * This is the drop-in boundary for k-wave-swift's
 *   kspaceFirstOrder(grid:medium:source:sensor:options:) -> SimulationOutput
 * (Sources/KWave/Solver/KSpaceFirstOrder.swift:79-107). A Swift `.systemLibrary` target
 * (modelled on Sources/CHDF5/module.modulemap:1-5) links this library; the Swift adapter
 * flattens its KWaveGrid / KWaveMedium / KWaveSource / KWaveSensor / SimulationOptions values
 * into one kw_sim_desc of plain host pointers, calls kw_sim_create + kw_sim_run, and copies the
 * SimulationOutput fields back with kw_sim_get_output.
 *
 * Conventions
 *   - Every function returns a kw_status (0 = KW_OK) and never aborts the process. The text of the
 *     last error of a context is kw_last_error_message(ctx). The reference traps on the same
 *     conditions (precondition/fatalError, KSpaceFirstOrder.swift:105,210-212,358-360,369-370;
 *     Recording.swift:76-77); here they come back as KW_ERR_INVALID.
 *   - All arrays are row-major (C order) float32 host arrays, last axis contiguous, exactly the
 *     memory order of an MLXArray of shape [nx], [nx, ny] or [nx, ny, nz]. The library copies
 *     every input during kw_sim_create; the caller keeps ownership of its buffers.
 *   - One kw_context per host thread; a context (and the sims/batches made from it) must not be
 *     used by two threads at once without external locking.
 *   - All device work of a context runs on one CUDA stream (its own, or the caller's stream set
 *     with kw_context_set_stream).
 */
#ifndef KWAVE_CUDA_H
#define KWAVE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KW_ABI_VERSION 2

#if defined(__GNUC__)
#define KW_API __attribute__((visibility("default")))
#else
#define KW_API
#endif

/* ---- status codes ------------------------------------------------------------------------ */
typedef enum kw_status {
    KW_OK = 0,
    KW_ERR_INVALID = 1,     /* a descriptor or argument the reference would reject (precondition) */
    KW_ERR_OOM = 2,         /* device or host allocation failed */
    KW_ERR_CUDA = 3,        /* a CUDA runtime call failed (message has the CUDA error string) */
    KW_ERR_NONFINITE = 4,   /* the pressure field became NaN/Inf (checked every few steps) */
    KW_ERR_TIMEOUT = 5,     /* a bounded device-side wait ran out */
    KW_ERR_UNSUPPORTED = 6, /* a size or mode this build does not implement (e.g. FFT length) */
    KW_ERR_STATE = 7        /* call out of order (e.g. output requested before kw_sim_run) */
} kw_status;

/* ---- enums mirroring the reference types ------------------------------------------------ */

/* SourceMode (Sources/KWave/Source/KWaveSource.swift:4-8). */
typedef enum kw_source_mode {
    KW_SOURCE_DIRICHLET = 0,
    KW_SOURCE_ADDITIVE = 1,               /* default in the reference */
    KW_SOURCE_ADDITIVE_NO_CORRECTION = 2
} kw_source_mode;

/* AbsorptionMode (Sources/KWave/Medium/KWaveMedium.swift:8-17). */
typedef enum kw_absorption_mode {
    KW_ABSORPTION_NONE = 0,               /* .noAbsorption (default) */
    KW_ABSORPTION_POWER_LAW = 1,          /* .powerLaw */
    KW_ABSORPTION_NO_DISPERSION = 2,      /* .noDispersion */
    KW_ABSORPTION_STOKES = 3              /* .stokes */
} kw_absorption_mode;

/* DirectivityPattern (Sources/KWave/Sensor/KWaveSensor.swift:24-29). */
typedef enum kw_directivity_pattern {
    KW_DIRECTIVITY_PRESSURE = 0,
    KW_DIRECTIVITY_GRADIENT = 1
} kw_directivity_pattern;

/* RecordField bit values, identical to Sources/KWave/Sensor/KWaveSensor.swift:4-21. */
#define KW_RECORD_P        (1u << 0)
#define KW_RECORD_P_MAX    (1u << 1)
#define KW_RECORD_P_MIN    (1u << 2)
#define KW_RECORD_P_RMS    (1u << 3)
#define KW_RECORD_P_FINAL  (1u << 4)
#define KW_RECORD_UX       (1u << 5)
#define KW_RECORD_UY       (1u << 6)
#define KW_RECORD_UZ       (1u << 7)
#define KW_RECORD_U_MAX    (1u << 8)
#define KW_RECORD_U_RMS    (1u << 9)
#define KW_RECORD_U_FINAL  (1u << 10)
#define KW_RECORD_I_AVG    (1u << 11)
#define KW_RECORD_I_MAX    (1u << 12)

/* Sensor mask kinds. The reference decides by shape (Recording.swift:50-56): a mask of shape
 * [dim, nPoints] is Cartesian, anything else is a binary grid mask. The caller passes the
 * decision explicitly. */
typedef enum kw_sensor_kind {
    KW_SENSOR_NONE = 0,
    KW_SENSOR_BINARY = 1,      /* grid-shaped mask, nonzero = sensor point */
    KW_SENSOR_CARTESIAN = 2    /* [dim][n_points] coordinates in metres, grid centre at n/2 */
} kw_sensor_kind;

/* SimulationOutput fields (KSpaceFirstOrder.swift:47-73). */
typedef enum kw_field {
    KW_FIELD_P = 0,          /* [nSensor, nt] */
    KW_FIELD_P_MAX,          /* [nSensor] */
    KW_FIELD_P_MIN,
    KW_FIELD_P_RMS,
    KW_FIELD_P_FINAL,        /* grid shape, always present */
    KW_FIELD_UX,             /* [nSensor, nt], collocated to the pressure grid */
    KW_FIELD_UY,
    KW_FIELD_UZ,
    KW_FIELD_UX_MAX,         /* [nSensor] */
    KW_FIELD_UY_MAX,
    KW_FIELD_UZ_MAX,
    KW_FIELD_UX_RMS,
    KW_FIELD_UY_RMS,
    KW_FIELD_UZ_RMS,
    KW_FIELD_UX_FINAL,       /* grid shape, staggered grid */
    KW_FIELD_UY_FINAL,
    KW_FIELD_UZ_FINAL,
    KW_FIELD_IX_AVG,         /* [nSensor] */
    KW_FIELD_IY_AVG,
    KW_FIELD_IZ_AVG,
    KW_FIELD_COUNT
} kw_field;

/* ---- descriptor ---------------------------------------------------------------------------- */

/* A float32 host array that is either a scalar (len == 1) or grid-shaped (len == nx*ny*nz).
 * data == NULL means "absent" (only meaningful for optional medium properties). */
typedef struct kw_array {
    const float* data;
    size_t len;
} kw_array;

/* A source signal: one broadcast row (rows == 1) or one row per source point (rows == nSrc,
 * in ascending flat mask order), each `len` samples long, row-major. data == NULL: absent. */
typedef struct kw_signal {
    const float* data;
    int rows;
    int len;
} kw_signal;

/* One simulation: the reference's grid, medium, source, sensor and options flattened.
 * Source line references are Sources/KWave/... paths of k-wave-swift. */
typedef struct kw_sim_desc {
    int abi_version;                 /* must be KW_ABI_VERSION */

    /* KWaveGrid (Grid/KWaveGrid.swift:9-101); unused sizes are 1. */
    int dim;                         /* 1, 2 or 3 */
    int nx, ny, nz;
    double dx, dy, dz;
    double dt;                       /* from makeTime / setTime (KWaveGrid.swift:112-142) */
    int nt;

    /* SimulationOptions (Solver/KSpaceFirstOrder.swift:17-40). dtype, device, pmlInside,
     * plotSim and saveToDisk are not read by the reference solver and have no field here. */
    int pml_size;                    /* PMLSize.uniform(n); the PML is inside the grid */
    double pml_alpha;                /* default 2.0 */
    int smooth_p0;                   /* default 1 */
    int smooth_c0;                   /* default 0 */
    int smooth_rho0;                 /* default 0 */
    double c_ref;                    /* NaN (default): max(c0) after smoothing, as the reference;
                                        otherwise this value (used by the adjoint, where cRef is
                                        held fixed) */

    /* KWaveMedium (Medium/KWaveMedium.swift:21-76). */
    kw_array sound_speed;            /* required */
    kw_array density;                /* required */
    kw_array alpha_coeff;            /* dB/(MHz^y cm); data == NULL: lossless */
    double alpha_power;              /* NaN: absent (the reference then uses 1.5) */
    int alpha_mode;                  /* kw_absorption_mode */
    kw_array b_on_a;                 /* data == NULL: linear */

    /* KWaveSource (Source/KWaveSource.swift:11-71). Elastic stress fields are not part of the
     * fluid solver and are not carried. */
    const float* p0;                 /* grid-shaped initial pressure or NULL */
    const float* p_mask;             /* grid-shaped or NULL */
    kw_signal p;
    int p_mode;                      /* kw_source_mode */
    const float* u_mask;             /* grid-shaped or NULL */
    kw_signal ux, uy, uz;
    int u_mode;                      /* kw_source_mode */

    /* KWaveSensor (Sensor/KWaveSensor.swift:32-62). */
    int sensor_kind;                 /* kw_sensor_kind */
    const float* sensor_mask;        /* grid-shaped (binary) or [dim][sensor_points] (Cartesian) */
    int sensor_points;               /* Cartesian point count (ignored for binary masks) */
    unsigned record;                 /* KW_RECORD_* bits; default KW_RECORD_P */
    const float* directivity_angle;  /* 2D binary sensors only: grid-shaped angles (rad) or NULL */
    double directivity_size;         /* NaN: 10*max(dx, dy) */
    int directivity_pattern;         /* kw_directivity_pattern */

    /* 1: run kspaceFirstOrderAS (Solver/KSpaceFirstOrderAS.swift:19-309) instead of
     * kspaceFirstOrder: 2D, x axial, y radial (r >= 0, PML at the outer edge only); p0 and
     * pressure / velocity sources, Stokes absorption, B/A; records p and pFinal. */
    int axisymmetric;
} kw_sim_desc;

/* Fill a descriptor with the reference's defaults (SimulationOptions(), KWaveSource(),
 * KWaveSensor()): pml 20, alpha 2, smoothP0 on, additive sources, record = KW_RECORD_P. */
KW_API void kw_sim_desc_init(kw_sim_desc* desc);

/* ---- callbacks ----------------------------------------------------------------------------- */

/* progress(t, nt): SimulationOptions.progress, called once per time step after the step has
 * been issued (KSpaceFirstOrder.swift:30-31,544). */
typedef void (*kw_progress_fn)(int t, int nt, void* user);
/* monitor(t, p, count): SimulationOptions.fieldMonitor, called every `monitor_interval` steps
 * with a host copy of the whole pressure field (KSpaceFirstOrder.swift:32-37,541-543). */
typedef void (*kw_monitor_fn)(int t, const float* p, size_t count, void* user);

typedef struct kw_callbacks {
    kw_progress_fn progress;
    kw_monitor_fn monitor;
    int monitor_interval;            /* <= 0 is treated as 1, like max(interval, 1) */
    void* user;
} kw_callbacks;

/* ---- opaque handles ------------------------------------------------------------------------ */
typedef struct kw_context kw_context;
typedef struct kw_sim kw_sim;
typedef struct kw_batch kw_batch;

/* ---- library / context --------------------------------------------------------------------- */
KW_API const char* kw_version(void);
KW_API int kw_abi_version(void);

/* Create a context on CUDA device `device` with its own non-blocking stream. */
KW_API int kw_context_create(int device, kw_context** out);
/* Run all further work of this context on `cuda_stream` (a cudaStream_t; NULL restores the
 * context's own stream). */
KW_API int kw_context_set_stream(kw_context* ctx, void* cuda_stream);
KW_API void kw_context_destroy(kw_context* ctx);
KW_API const char* kw_last_error_message(const kw_context* ctx);

/* ---- one simulation: kspaceFirstOrder ------------------------------------------------------ */

/* Validate the descriptor, run the once-per-run setup (smoothing, operators, PML, source and
 * sensor plans; KSpaceFirstOrder.swift:351-490) and upload everything to the device. */
KW_API int kw_sim_create(kw_context* ctx, const kw_sim_desc* desc, kw_sim** out);
/* Run all nt time steps from t = 0 (resets the state first) and finalise the recording
 * (KSpaceFirstOrder.swift:492-554). `cb` may be NULL. */
KW_API int kw_sim_run(kw_sim* sim, const kw_callbacks* cb);
/* Reset the state to t = 0 without running. */
KW_API int kw_sim_reset(kw_sim* sim);
/* Advance `nsteps` further time steps (clamped to nt) without callbacks; asynchronous on the
 * context's stream. Used for incremental runs and timing. */
KW_API int kw_sim_step(kw_sim* sim, int nsteps);
/* Block until all issued work has finished; reports KW_ERR_NONFINITE if p became non-finite. */
KW_API int kw_sim_synchronize(kw_sim* sim);
/* Current time index (number of steps taken since the last reset). */
KW_API int kw_sim_current_step(const kw_sim* sim, int* t);
KW_API int kw_sim_num_sensor_points(const kw_sim* sim, int* count);
/* Element count of an output field (0 when the field was not requested / does not apply). */
KW_API int kw_sim_output_size(const kw_sim* sim, int field, size_t* count);
/* Copy an output field into `dst` (count must equal kw_sim_output_size). Series are
 * [nSensor, nt] row-major over the steps taken so far. */
KW_API int kw_sim_get_output(kw_sim* sim, int field, float* dst, size_t count);
/* Device pointer of a live state field (KW_FIELD_P_FINAL = p, KW_FIELD_U?_FINAL = u) for
 * zero-copy consumers such as a field monitor; valid until the next step. */
KW_API int kw_sim_device_field(kw_sim* sim, int field, const float** dptr, size_t* count);
KW_API void kw_sim_destroy(kw_sim* sim);

/* ---- measurement ---------------------------------------------------------------------------
 * The reference has no profiler (its bench wall-clocks whole runs, Sources/KWaveBench/main.swift:
 * 50-57). This entry point runs `reps` further time steps launch by launch with CUDA events around
 * every launch and reports, for each launch of one step in issue order, its mean device time and
 * its algorithmic HBM bytes (the compulsory reads + writes of that pass). */
typedef struct kw_kernel_timing {
    char name[48];       /* "<pass>:<job>", e.g. "colA_op:vel", "c2r:den" */
    double ms;           /* mean device time per launch */
    double bytes;        /* algorithmic HBM bytes per launch */
} kw_kernel_timing;
KW_API int kw_sim_profile_step(kw_sim* sim, int reps, kw_kernel_timing* out, int max_entries, int* n_entries);

/* ---- standalone spectral operator ------------------------------------------------------------
 * Staggered spectral derivative of one device field along `axis` (0 = x):
 *   out = Re F^-1( i k exp(shift * i k d/2) F(in) ),  shift = +1 or -1,
 * the reference's derivativeOperator (Solver/KSpaceFirstOrder.swift:764-769) applied on its own
 * (the time step also multiplies by kappa). d_in and d_out are device pointers to nx*ny*nz
 * row-major floats (unused sizes 1) and may not overlap. Runs on the context's stream and returns
 * after the result is written. The half-spectrum scratch is allocated and freed inside the call. */
KW_API int kw_spectral_derivative(kw_context* ctx, int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                                  int axis, int shift, const float* d_in, float* d_out);

/* Allocation-free variant of kw_spectral_derivative (no counterpart in the reference). Same
 * arguments and result; it never calls cudaMalloc or cudaFree. It is for callers that cannot
 * allocate device memory: a host whose own memory manager already holds the device memory, or a
 * loop that cannot take cudaMalloc/cudaFree's device-wide synchronisation. Its scratch (the
 * half-spectrum, twiddle tables, operator vector, tile maps) lives in one file-scope device array
 * of KW_NOALLOC_SCRATCH_BYTES that every GPU loading this library keeps until the process exits;
 * problems that need more are rejected with KW_ERR_INVALID and a message naming the limit (about
 * 2 M half-spectrum values: e.g. 2D 1024^2 or 3D 128^3 fit). Every call looks up the array's
 * device address (cudaGetSymbolAddress) with the context's device current, so a device whose
 * context was reset and re-created is served from its new copy. All calls share the array and it
 * keeps the last call's contents (each call clears what it uses); calls whose work overlaps on the
 * GPU race on it. */
#define KW_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
KW_API int kw_spectral_derivative_noalloc(kw_context* ctx, int dim, int nx, int ny, int nz, double dx, double dy,
                                          double dz, int axis, int shift, const float* d_in, float* d_out);

/* ---- many independent simulations in one launch sequence -----------------------------------
 * Simulations of the same dimensionality (any sizes, any nt) step together: every kernel of a
 * step covers the tiles of all simulations that are still running, so small grids fill the GPU.
 * Each member behaves exactly as kw_sim_run would for its own descriptor. */
KW_API int kw_batch_create(kw_context* ctx, const kw_sim_desc* descs, int count, kw_batch** out);
KW_API int kw_batch_run(kw_batch* batch, const kw_callbacks* cb);
KW_API int kw_batch_reset(kw_batch* batch);
KW_API int kw_batch_step(kw_batch* batch, int nsteps);
KW_API int kw_batch_synchronize(kw_batch* batch);
KW_API int kw_batch_output_size(const kw_batch* batch, int index, int field, size_t* count);
KW_API int kw_batch_get_output(kw_batch* batch, int index, int field, float* dst, size_t count);
KW_API void kw_batch_destroy(kw_batch* batch);

/* ---- adjoint gradient of a sensor-data misfit --------------------------------------------------
 * Gradients of L = 1/2 sum_t sum_q (p_q(t) - data_q(t))^2 (p_q: the pressure the forward
 * kw_sim_run records at sensor point q) with respect to the sound speed c0 and the density rho0
 * (one value per grid point; a scalar c0 or rho0 is differentiated as a uniform map, whose
 * scalar derivative is the sum of the field) and the initial pressure p0, by the exact discrete
 * adjoint of the time step: every operator of the step transposed in reverse order. The reference has no adjoint; this is the
 * kspaceFirstOrderAdjoint entry a Swift adapter would expose next to kspaceFirstOrder
 * (Sources/KWave/Solver/KSpaceFirstOrder.swift:79-107 is the forward it differentiates).
 * The reverse sweep needs the forward states in reverse order; they are recomputed segment by
 * segment from checkpoints (policy below). c_ref (kappa, PML) and dt are held fixed.
 * Supported: 1D/2D/3D, heterogeneous c0/rho0, lossless / Stokes / power law (with or without
 * dispersion), B/A, source.p0 and k-space corrected additive pressure sources, binary or
 * Cartesian sensors. KW_ERR_UNSUPPORTED: velocity sources, Dirichlet or uncorrected pressure
 * sources, directivity, smoothC0 / smoothRho0 maps, grad_p0 with smoothP0. */
typedef enum kw_checkpoint_policy {
    KW_CHECKPOINT_SQRT = 0,      /* ceil(sqrt(nt)) steps between checkpoints, segments recomputed */
    KW_CHECKPOINT_INTERVAL = 1,  /* checkpoint_interval steps between checkpoints */
    KW_CHECKPOINT_BUDGET = 2,    /* keep every state when that fits memory_budget bytes, else the
                                    interval that needs the least memory */
    KW_CHECKPOINT_STORE_ALL = 3, /* keep every state of the forward run (no recompute) */
    KW_CHECKPOINT_REVOLVE = 4    /* binomial (revolve) schedule: checkpoint_interval > 0 snapshots of
                                    the state, else as many as memory_budget holds; one tape slot;
                                    a step is recomputed at most r times, r the least with
                                    C(snapshots + r, r) >= nt (BUDGET falls back to it when no
                                    uniform interval fits the budget) */
} kw_checkpoint_policy;

typedef struct kw_adjoint_desc {
    int abi_version;              /* KW_ABI_VERSION */
    const float* data;            /* observed sensor pressure [n_sensor][nt], the p output's layout */
    int policy;                   /* kw_checkpoint_policy */
    int checkpoint_interval;      /* KW_CHECKPOINT_INTERVAL */
    double memory_budget;         /* KW_CHECKPOINT_BUDGET, bytes of device memory for states */
    float* grad_c0;               /* out: dL/dc0 on the grid (same layout as sound_speed), or NULL */
    float* grad_p0;               /* out: dL/dp0 on the grid, or NULL (needs source.p0) */
    float* grad_rho0;             /* out: dL/drho0 on the grid, or NULL (rho0 enters dt rho0 nl,
                                     dt / staggerDensity(rho0), rho0 div and B/A S^2 / (2 rho0)) */
    double misfit;                /* out: L */
    double forward_ms;            /* out: device time of the forward run that stores checkpoints */
    double reverse_ms;            /* out: device time of the reverse sweep (recompute included) */
    int interval;                 /* out: steps between checkpoints actually used */
    int checkpoints;              /* out: stored checkpoints (0 when every state was kept) */
} kw_adjoint_desc;

KW_API void kw_adjoint_desc_init(kw_adjoint_desc* adj);
KW_API int kw_adjoint_run(kw_context* ctx, const kw_sim_desc* desc, kw_adjoint_desc* adj);

#ifdef __cplusplus
}
#endif

#endif /* KWAVE_CUDA_H */
