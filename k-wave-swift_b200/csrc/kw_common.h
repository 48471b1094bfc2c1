// kw_common.h — structures shared by the host engine and the sm_100a kernels.
//
// Layout. Every simulation stores its real fields as [A][B][C] float32 with C contiguous:
//   1D (nx):        A = 1,  B = 1,  C = nx
//   2D (nx, ny):    A = 1,  B = nx, C = ny
//   3D (nx,ny,nz):  A = nx, B = ny, C = nz
// i.e. exactly the row-major order of the reference's MLXArray fields. Spectra are the
// half-spectrum of a real transform along C: [A][B][Cp] float2 with Ch = C/2 + 1 bins per row,
// padded to Cp = Ch rounded up to a multiple of 4, so that every spectrum row and every row of a
// float table over the half spectrum starts 16-byte aligned (TMA strides). Padding bins hold zeros.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace kw {

constexpr int kMaxStages = 16;
constexpr int kMaxComp = 3;
constexpr int kAdjFields = 32;
constexpr int kMaxDirAngles = 16;   // distinct 2D sensor directivity angles of one simulation

// FFT plan of one complex transform length n (a Stockham sequence of radix stages).
struct FFTPlanDev {
    int n;
    int nstages;
    int radix[kMaxStages];
    int tw_off[kMaxStages];   // offset of stage s in `tw` (Ns*(R-1) entries, forward sign)
    const float2* tw;         // exp(-2 pi i r k / (Ns R)), k in [0, Ns), r in [1, R)
    const float2* gen;        // for generic-prime stages: exp(-2 pi i m / R) at tw_off-independent offsets
    int gen_off[kMaxStages];
    const float2* twn;        // W_n^m = exp(-2 pi i m / n), m < n (compile-time specialised kernels)
};

// Lines per CTA of the pass kernels, shared by the host (tile maps, shared-memory sizes) and the
// kernels. Row passes stage L rows of M = C/2 complex values; column passes stage L columns of
// length N.
// About 4096 complex values per tile: short lines are batched 32 to a CTA, long ones 2.
__host__ __device__ constexpr int tile_lines(int n) {
    return n <= 128 ? 32 : (n <= 256 ? 16 : (n <= 512 ? 8 : (n <= 1024 ? 4 : 2)));
}
__host__ __device__ constexpr int row_lines(int M) { return tile_lines(M); }
__host__ __device__ constexpr int col_lines(int N) { return tile_lines(N); }
// operator (fwd -> H -> inv) column passes keep an extra work tile and the staged radial table
__host__ __device__ constexpr int col_lines_op(int N) { return tile_lines(N) > 2 ? tile_lines(N) / 2 : 2; }
// C2R passes also stage their epilogue inputs, so they take half as many lines
__host__ __device__ constexpr int c2r_lines(int M) { return tile_lines(M) > 2 ? tile_lines(M) / 2 : 2; }

// Register-resident transforms (kw_fft_reg.cuh): lengths with a register plan are the powers of
// two 16 ... 4096 and 12 * 2^k, 24 ... 3072. N / R1 threads hold R1 values each, so one 256-thread
// group covers 256 / (N / R1) lines. The in-place column passes (TMA-fed, kw_pass_colp.cu) take
// lengths up to 256 (one TMA box), the operator column pass (kw_pass_colop.cu) up to 1024, the row
// passes (kw_pass_rowr.cu) half lengths up to 2048.
__host__ __device__ constexpr bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
__host__ __device__ constexpr bool has_reg_plan(int n) {
    return (is_pow2(n) && n >= 16 && n <= 4096) || (n % 12 == 0 && is_pow2(n / 12) && n / 12 >= 2 && n / 12 <= 256);
}
__host__ __device__ constexpr int reg_r1(int n) { return n % 3 == 0 ? 12 : (n >= 128 ? 16 : (n >= 32 ? 8 : 4)); }
__host__ __device__ constexpr int reg_lines(int n, int r1) { return 256 / (n / r1); }
__host__ __device__ constexpr bool has_colp(int n) { return has_reg_plan(n) && n <= 256; }
__host__ __device__ constexpr bool has_colop(int n) { return has_reg_plan(n) && n <= 1024; }
__host__ __device__ constexpr int colr_lines(int n) { return reg_lines(n, reg_r1(n)); }
__host__ __device__ constexpr int colop_lines(int n) { return reg_lines(n, reg_r1(n)); }
// Row passes for even rows: R2C threads hold reg_r1(M) values; C2R threads, whose epilogues keep
// more state, hold c2r_r1(M) (more threads per row, fewer registers each).
__host__ __device__ constexpr bool has_reg_row(int M) { return has_reg_plan(M) && M <= 2048; }
__host__ __device__ constexpr int c2r_r1(int M) { return M % 3 == 0 ? 12 : (M <= 16 ? 4 : 8); }
__host__ __device__ constexpr int r2c_rows(int M) { return reg_lines(M, reg_r1(M)); }
__host__ __device__ constexpr int c2r_rows(int M) { return reg_lines(M, c2r_r1(M)); }

// size lists of the instantiated register-plan kernels
#define KW_REG_ROW_SIZES(X) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(2048) X(24) X(48) X(96) X(192) X(384) \
    X(768) X(1536)
#define KW_COLP_SIZES(X) X(16) X(32) X(64) X(128) X(256) X(24) X(48) X(96) X(192)
#define KW_COLOP_SIZES(X) X(16) X(32) X(64) X(128) X(256) X(512) X(1024) X(24) X(48) X(96) X(192) X(384) X(768)

// Line lengths with compile-time specialised pass kernels (in-place, one shared buffer per tile);
// every other length runs the runtime-plan kernels (ping-pong, two buffers per tile).
#define KW_FFT_SIZES(X) X(8) X(12) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) \
    X(512) X(768) X(1024)
__host__ __device__ constexpr bool has_fixed_kernel(int n) {
#define KW_IS(m) n == m ||
    return KW_FFT_SIZES(KW_IS) false;
#undef KW_IS
}

// Per-axis operator vectors in FFT order (length n of that axis). Each is already made
// Hermitian (real part at the Nyquist bin), so Re(ifft(H * fft(x))) == C2R(H * R2C(x)).
struct AxisDev {
    int n;
    const float2* dpos;     // i k exp(+i k d/2)
    const float2* dneg;     // i k exp(-i k d/2)
    const float2* colloc;   // exp(-i k d/2)
    const float* pml;       // collocated PML profile
    const float* pml_sg;    // staggered PML profile
    float inv_d;            // 1 / spacing
};

// A float32 quantity that is either one value or a full [A][B][C] field.
struct FieldOrScalar {
    const float* ptr;       // nullptr: use `s`
    float s;
    __host__ __device__ float at(long long i) const { return ptr ? ptr[i] : s; }
};

// Radial (|k|-only) operator tables over the half-spectrum [A][B][Cp], precomputed in FP64.
// RT_DIR0 + j: the k-space weight of directivity angle j (Hermitian part; [A][B][Cp])
enum RadialTable { RT_NONE = 0, RT_KAPPA, RT_SKAPPA, RT_NU1, RT_NU2, RT_WINDOW, RT_DIR0, RT_COUNT = RT_DIR0 + kMaxDirAngles };
// Per-axis factor selector.
enum AxisOp { AO_NONE = 0, AO_DPOS, AO_DNEG, AO_COLLOC };

struct OpSpec {
    int8_t axis_op;   // AxisOp
    int8_t axis;      // reference axis (0 = x) the per-axis factor applies to
    int8_t radial;    // RadialTable
    int8_t src;       // input component this output reads
};

// Epilogues of the inverse row pass (C2R), i.e. what happens to the inverse-transformed
// values d_o of the job's outputs o at each grid point.
enum Epilogue {
    EPI_STORE = 0,       // out_field[o][i] = d_o
    EPI_VEL,             // u_a = pml_sg_a (pml_sg_a u_a - dtor_a d_a)             (velStep)
    EPI_VEL_INIT,        // u_a = 0.5 dtor_a d_a                                    (t = 0 override)
    EPI_DEN,             // nl; rho_a = pml_a (pml_a rho_a - dtrho0 d_a nl); rho_sum; div; EoS
    EPI_ADD_U,           // u_{comp(o)} += d_o                                       (additive u source)
    EPI_ADD_RHO,         // rho_a += d_0 / d_a; rho_sum; EoS                          (additive p source)
    EPI_EOS_ABS,         // p = c2 (rho_sum + tau d_0 - eta d_1 + nonlinear)          (power law)
    // discrete adjoint (kw_adjoint.cpp; register row kernels only)
    EPI_ADJ_VEL,         // mu = lambda_u_a - d_a; lambda_u_a = sg_a^2 mu; w_a = sg_a dtor_a mu
    EPI_ADJ_SUM,         // lambda_p = sum_a d_a; x1 = tau c2 lambda_p; x2 = eta c2 lambda_p
    EPI_ADJ_EOS,         // the reverse equation of state (kw_adjoint.cu k_adj_eos) with d = A1, A2, A2(S)
    EPI_DEN_SRC,         // EPI_DEN + rho_a += signal[t] psrc_q / d_a (precorrected pressure source active)
    EPI_ADJ_EOS_RHO,     // EPI_ADJ_EOS + the direct terms of dL/drho0
    EPI_ADJ_VEL_RHO,     // EPI_ADJ_VEL + dL/d(dt / rho_sg_a) += -sg_a g_a mu (density gradient)
};

// Source operator of one field variable (SourceOp, KSpaceFirstOrder.swift:129-175).
struct SourceDev {
    int nsrc;
    int rows;              // 1 (broadcast) or nsrc
    int len;               // samples
    int mode;              // kw_source_mode
    const int* idx;        // [nsrc] flat indices, ascending
    const float* signal;   // [rows][len]
    const float* scale[kMaxComp];  // per-axis (p) or per-component (u) per-point scale, [nsrc]
};

struct SensorDev {
    int kind;              // 0 none, 1 binary, 2 cartesian
    int npts;
    int ncorners;
    const int* idx;        // [npts * ncorners]
    const float* w;        // [npts * ncorners] (cartesian)
    int record_p_series;   // keep p[t][q]
    int record_u_series;   // keep u[a][t][q]
    int record_p_agg;      // running max/min/sum-of-squares of p
    int record_u_agg;
    float* p_series;       // [nt][npts]
    float* u_series[kMaxComp];
    float* p_max; float* p_min; float* p_ss; float* p_ssc;   // running aggregates (Kahan)
    float* u_max[kMaxComp]; float* u_ss[kMaxComp]; float* u_ssc[kMaxComp];
    // 2D directivity (binary sensors): p of row q is sampled from dir_field[dir_slot[q]], the
    // pressure filtered by the k-space weight of the row's angle ([ndir][N])
    int ndir;
    float* dir_field;
    const int* dir_slot;
};

// Tensor maps of one simulation (TMA descriptors, kw_tmaps.cpp): spectrum s viewed as tiles of
// pass-axis lines for layout axis A (2D view [A][B*Cp]) or B (3D view [A][B][Cp]); only the views
// an in-place column pass of a register-plan length needs are encoded.
__host__ __device__ constexpr int tmap_spec(int s, int layout_axis) { return 2 * s + layout_axis; }
constexpr int kNumTmaps = 8;

// Where the adjoint's reverse sweep finds the forward quantities of step t (one entry per step,
// device memory; kw_adjoint.cpp). Recomputed steps write it from their epilogues.
struct AdjTapeEntry {
    float* p;
    float* s;              // S(t) = sum_a rho_a
    float* sprev;          // S(t-1)
    float* div;            // Stokes div term
    float* dd[kMaxComp];   // d_a(t) = D-_a u_a(t) (B/A, or the density gradient)
    float* q2;             // A2(S(t)) (power law with dispersion)
    float* pprev;          // p(t-1) (density gradient)
};

struct SimDev {
    int dim;
    int A, B, C, Ch, Cp;
    long long N;           // real points A*B*C
    long long Ns;          // spectrum elements A*B*Cp
    int nt;
    int axis_of_layout[3]; // reference axis of layout axis A, B, C (-1 when the layout axis is 1)
    AxisDev ax[3];         // reference axes
    FFTPlanDev plan_row;   // complex plan of the row transform (length C/2 for even C, C for odd)
    const float2* row_tw;  // exp(-2 pi i k / C), k in [0, C/2]
    FFTPlanDev plan_b;     // column plan along B (length B)
    FFTPlanDev plan_a;     // column plan along A (length A)
    float inv_n;           // 1 / N
    const float* radial[RT_COUNT];   // [A][B][Cp] tables (nullptr when unused)
    const CUtensorMap* tmaps;        // [kNumTmaps] (device memory, 64-byte aligned)

    // state
    float* p;
    float* u[kMaxComp];
    float* rho[kMaxComp];
    float* rho_sum;
    float* div_term;       // rho0 * sum_a d_a (power law input) or sum_a d_a * tau * rho0 (Stokes)
    float* src_buf[kMaxComp];   // sparse scratch fields for additive sources (zero off-mask)
    float* tmp[kMaxComp];       // real scratch fields (collocated velocity etc.)
    float2* spec[4];
    float* adj[kAdjFields];     // adjoint work fields (kw_adjoint.cpp), unused by a forward run
    const AdjTapeEntry* tape;   // adjoint recompute: the tape epilogues store into tape[t] (else null)
    double* adj_gc;             // adjoint: dL/dc accumulated in FP64
    double* adj_gr;             // adjoint: the direct terms of dL/drho0 in FP64 (null: not requested)
    double* adj_gdtor[kMaxComp];   // adjoint: dL/d(dt / rho_sg_a) in FP64 (with adj_gr)
    int* adj_rev;               // adjoint: the reverse step counter
    float adj_y;                // adjoint: absorption power y

    // medium
    float dt;              // time step (FP32, multiplies rho0 like the reference's dt * rho0)
    FieldOrScalar c2, rho0, tau, eta, bona;
    FieldOrScalar dtor[kMaxComp];
    int nonlinear;
    int absorb;            // 0 none, 1 Stokes, 2 power law without dispersion, 3 with dispersion
    int eos_pointwise;     // EoS evaluated in the density epilogue / source kernels

    SourceDev psrc, usrc[kMaxComp];
    // Additive pressure source with one signal row: the k-space corrected source of step t is
    // signal[t] * Re F^-1(cos(c_ref dt k / 2) F(scale * mask)) (linearity; SourceOp.apply,
    // KSpaceFirstOrder.swift:167-172), so that field is computed once at setup and the density
    // epilogue adds signal[t] * psrc_q / d_a to each rho_a while the signal lasts (else null).
    const float* psrc_q;
    int has_p, has_u[kMaxComp];
    int has_p0;
    SensorDev sensor;
    int* nonfinite;        // device flag
    long long wait_cycles; // limit of a column pass consumer's wait for its tile (clock64 cycles)
    int test_stall;        // test hook: the TMA column pass withholds its first tile copy
};

// One entry of a launch's block map: which simulation, which component, which tile.
struct BlockWork {
    int sim;
    int comp;
    int tile;
};

}  // namespace kw
