// kw_kernels.cuh — launch-side descriptions of the sm_100a kernels (host and device).
#pragma once

#include "kw_common.h"

namespace kw {

// Which real field a pass reads or writes.
enum FieldSel {
    FS_P = 0, FS_U, FS_RHO, FS_RHO_SUM, FS_DIV, FS_SRCBUF, FS_TMP,
    FS_WORK,  // power-law absorption inputs: component 0 = rho0 div u, component 1 = rho_sum
    FS_ADJ    // adjoint work fields: FS_ADJ + k selects adj[k + component]
};
// FS_DIR + j: the directivity-filtered pressure of angle j + component (kw_common.h SensorDev)
constexpr int FS_DIR = FS_ADJ + kAdjFields;

// A launch may be gated on a source being active at the current step.
// GATE_DIR + j: open while the simulation has a directivity angle j.
enum Gate { GATE_NONE = 0, GATE_PSRC, GATE_USRC, GATE_P0, GATE_ABS, GATE_RECU, GATE_DIR = 16 };

enum ColMode { COL_FWD = 0, COL_INV, COL_FWD_OP_INV };

struct RowR2CJob {
    int in_field;          // FieldSel (component = BlockWork.comp)
    int spec_out;          // component c -> spec[spec_out + c]
    int apply_op;          // 1D: the row transform is the last forward pass
    OpSpec op[kMaxComp];
    int gate;
    long long tile_elems;  // float2 elements of one staged tile (max over the launch's simulations)
    int ahead;             // register rows: > 0, prefetch into L2 the input rows of the CTA this many entries on
};

struct ColJob {
    int layout_axis;       // 0 = A, 1 = B
    int mode;              // ColMode
    int spec_in;           // component c (or fan-out input) spec index
    int spec_out;
    int nout;              // outputs written by one CTA (fan-out) or 1
    int fanout;
    int fanin;             // > 0: the operator pass sums op[c] X_c over this many inputs into one output
    OpSpec op[kMaxComp];
    int gate;
    long long tile_elems;
    int tma_ahead;         // TMA column pass: > 0, also prefetch into L2 the tile this many of its tiles on
};

struct RowC2RJob {
    int spec_in;           // output o reads spec[spec_in + o]
    int ncomp;             // outputs handled by one CTA
    int epi;               // Epilogue
    int out_field;         // FieldSel for EPI_STORE
    int gate;
    int generic;           // some simulation needs the runtime-plan (ping-pong) path
    long long tile_elems;
    int tape;              // the density / source / absorption epilogues also fill the adjoint tape
    int prefetch;          // register row kernels: bulk-prefetch the CTA's rows of the epilogue's fields into L2
    int ahead;             // > 0: also the spectrum rows of the CTA this many map entries on (the next wave)
    int fwd;               // register row kernels: also run the forward R2C of the epilogue's output
    int fwd_spec;          // ... into spec[fwd_spec + o] (velocity: o = component; density: 0 = rho0 div u, 1 = rho_sum)
};

// Host entry points (kw_passes.cu, kw_small.cu). The pass launchers take the tile map and its
// length; the grid is persistent.
// `size_class` is the line length of the launch's simulations when it has a specialised kernel
// (has_fixed_kernel), else 0 (runtime plan).
void init_kernel_attributes();
void init_r2c_attributes(int optin);
void init_col_attributes(int optin);
void init_c2r_attributes(int optin);
void launch_row_r2c(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                    const RowR2CJob& job, size_t smem, int size_class);
void launch_col(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                const ColJob& job, size_t smem, int size_class);
void launch_row_c2r(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                    const RowC2RJob& job, size_t smem, int size_class);
// register-resident operator column pass for has_colop(n) lengths; one CTA per map entry,
// whose tile indexes colop_tile(n, v.r1) consecutive columns (the pass's outer extent is 1).
// A variant fixes the values per thread (r1) and the launch bound in CTAs per SM (minb, 0: none);
// colop_variants lists those of length n, the default first.
struct ColopVariant {
    int r1;
    int minb;
};
__host__ __device__ constexpr int colop_tile(int n, int r1) { return reg_lines(n, r1); }
// minb of the TMA-fed, warp-specialised variant (kw_pass_colop.cu): 3D operator passes along A of
// the lengths colop_tma_length(n) whose simulations have the A-axis tensor maps (r1 = 16)
constexpr int kColopTma = -1;
constexpr int kColopPf = -10;   // persistent L2-prefetching variants: minb = kColopPf - CTAs per SM
bool colop_tma_length(int n);
int colop_variants(int n, ColopVariant* out, int max);
void init_colop_attributes(int optin);
void launch_colop(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                  const ColJob& job, int n, ColopVariant v, int* err = nullptr);
// axisymmetric solver (kw_axisym.cu): radial mirror of an [nx][ny] field into the [nx][4 ny]
// expansion (WSWA: p, ux; HAHS: uy; HSHA: uy / r with over_r), the trimmed updates, sources
enum AsMirror { AS_WSWA = 0, AS_HAHS, AS_HSHA };
void launch_as_mirror(cudaStream_t st, const SimDev* std_sim, const SimDev* car, long long n_exp, const float* src,
                      float* dst, int kind, int over_r);
void launch_as_vel(cudaStream_t st, const SimDev* std_sim, long long n, const float* g0, const float* g1, int nye, int init);
void launch_as_den(cudaStream_t st, const SimDev* std_sim, long long n, const float* d0, const float* d1, const float* d2,
                   int nye);
void launch_as_eos(cudaStream_t st, const SimDev* std_sim, long long n);
void launch_as_p0(cudaStream_t st, const SimDev* std_sim, long long n, const float* p0);
void launch_as_src(cudaStream_t st, const SimDev* std_sim, const int* d_t, int nsrc, int target, float* buf);
void launch_as_add(cudaStream_t st, const SimDev* std_sim, long long n, const float* g, int nye, float* f0, float* f1);
// persistent, cp.async double-buffered register column passes for has_colop(n) lengths: in-place
// forward / inverse, operator (with fan-out) and fan-in operator modes; same tiles as launch_colop
// (colop_lines(n) consecutive columns of one plane)
enum ColaMode { CA_FWD = 0, CA_INV, CA_OP, CA_FANIN };
void init_cola_attributes(int optin);
void launch_cola(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                 const ColJob& job, int n);
// TMA-fed warp-specialised in-place column pass for has_colp(n) lengths (persistent grid);
// tiles are colr_lines(n) columns of one plane; `err` receives a KernelError code if a wait times out
void init_colp_attributes();
void launch_colp(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                 const ColJob& job, int n, int* err);
// register-resident row passes for even rows with has_reg_row(M) half lengths; one CTA per map
// entry, whose tile indexes r2c_rows(M) / c2r_rows(M) consecutive rows
void init_rowr_attributes(int optin);
// 3D plane pass on a thread-block cluster (kw_pass_plane.cu): R2C along C and the forward FFT along
// B of whole A-planes, map entries (sim, comp, plane a); plane_cluster(M, B) is the cluster size of
// the instantiated (half row length, column length) pairs, 0 when there is none
int plane_cluster(int M, int NB);
void init_plane_attributes(int optin);
void launch_plane_r2c(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                      const RowR2CJob& job, int M, int NB);
void launch_rowr_r2c(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                     const RowR2CJob& job, int M);
void launch_rowr_c2r(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                     const RowC2RJob& job, int M);

// small kernels: one block row per simulation (map entries with tile = block index in sim)
void launch_init_p0(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nblocks,
                    const float* const* d_p0s);
void launch_src_u(cudaStream_t st, const SimDev* d_sims, const int* d_t, int nsims, int max_src, int scatter_only);
void launch_src_p(cudaStream_t st, const SimDev* d_sims, const int* d_t, int nsims, int max_src, int scatter_only);
// tick_count (a zeroed device counter): the launch also advances the step counter *d_t once every
// CTA has read it, for a sample that is the last launch of the step
void launch_sample(cudaStream_t st, const SimDev* d_sims, int* d_t, int nsims, int max_pts, int which, int comp,
                   unsigned int* tick_count = nullptr);
void launch_tick(cudaStream_t st, int* d_t);
void launch_scatter(cudaStream_t st, float* dst, const int* idx, const float* val, int n);
void launch_check_finite(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nblocks);

// once-per-simulation setup on the device in FP64 (kw_setup.cu)
void launch_setup_c2(cudaStream_t st, const float* c0, float* c2, long long n);
void launch_setup_dtor(cudaStream_t st, const float* rho0, float* out, long long n, long long stride, int len, double dt);
void launch_setup_absorb(cudaStream_t st, const float* c0_map, double c0_s, const float* alpha_map, double alpha_s,
                         double np1, double y, int stokes, double tn, float* tau, float* eta, long long n);
void launch_setup_radial(cudaStream_t st, const double* kA, const double* kB, const double* kC, int A, int B, int Ch,
                         int Cp, double half, double y, float* kap, float* skap, float* nu1, float* nu2);
// largest value of x as order-preserving bits (atomicMax into *d_bits, zeroed by the caller) and
// its decoding
void launch_setup_max(cudaStream_t st, const float* x, long long n, unsigned int* d_bits);
float setup_max_decode(unsigned int bits);

// setup helpers on one field (single simulation)
void launch_absmax(cudaStream_t st, const float* x, long long n, unsigned int* d_out_bits);
void launch_scale(cudaStream_t st, float* x, long long n, const unsigned int* d_num_bits, const unsigned int* d_den_bits);
void launch_intensity(cudaStream_t st, const float* p_series, const float* u_series, int nt_used, int npts,
                      const float* h, float* out);

}  // namespace kw
