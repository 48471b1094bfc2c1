// kw_adjoint.h — shared declarations of the discrete adjoint (kw_adjoint.cu, kw_adjoint.cpp).
#pragma once

#include "kw_kernels.cuh"

namespace kw {

// adjoint work fields of one simulation (SimDev::adj), addressed by the spectral jobs as
// FS_ADJ + index; inputs and outputs of one job are consecutive so that component c maps to
// index + c
enum AdjField {
    ADJ_LU = 0,       // lambda_u[a], 3
    ADJ_LR = 3,       // lambda_rho[a], 3
    ADJ_LP = 6,       // lambda_p
    ADJ_W = 7,        // w[a] (job inputs), 3
    ADJ_E = 10,       // e[a] (job outputs), 3
    ADJ_X1 = 13,      // tau c^2 lambda_p      } absorption job inputs: NU1, NU2
    ADJ_X2 = 14,      // eta c^2 lambda_p      }
    ADJ_STP = 15,     // S(t) (points into the tape)
    ADJ_A1 = 16,      // A1(tau c^2 lambda_p)  } outputs
    ADJ_A2 = 17,      // A2(eta c^2 lambda_p)  }
    ADJ_Q2 = 18,      // A2(S(t)) (points into the tape)
    ADJ_SIG = 19,     // sum_a L_a / dx_a
    ADJ_GSIG = 20,    // G(sigma)
    ADJ_DDP = 21,     // d_a(t) = D-_a u_a(t) (points into the tape), 3
    ADJ_GP = 24,      // g_a = D+_a p(t-1), the velocity update's pressure gradient (density gradient), 3
    ADJ_PTP = 27,     // p(t)   (points into the tape)
    ADJ_SPRP = 28,    // S(t-1) (points into the tape, a checkpoint or a zero field)
    ADJ_DIVP = 29,    // div(t) (points into the tape; Stokes)
    ADJ_PPREV = 30,   // p(t-1) (points into the tape, a checkpoint or a zero field; density gradient)
    ADJ_COUNT = 31
};
// entries that point into the tape instead of owning a field
__host__ __device__ constexpr bool adj_is_view(int k) {
    return k == ADJ_STP || k == ADJ_Q2 || (k >= ADJ_DDP && k < ADJ_DDP + 3) || k == ADJ_PTP || k == ADJ_SPRP ||
           k == ADJ_DIVP || k == ADJ_PPREV;
}

static_assert(ADJ_COUNT <= kAdjFields, "adjoint fields");

// device pointers of one reverse step
struct AdjStepArgs {
    const float* a1;
    const float* a2;
    float* lam_p;
    float* lam_u[kMaxComp];
    float* lam_r[kMaxComp];
    float* w[kMaxComp];
    const float* e[kMaxComp];
    float* sig;       // nullptr when no additive source is active at this step
    double* gc;
    float y;          // absorption power
};

void launch_set_step(cudaStream_t st, int* d_t, int t);
// A reverse step reads its step t from *d_rev (k_adj_eos counts it down), so that the same
// launches (a CUDA graph) serve every step. k_adj_begin sets the step counter *d_t = t, points the
// tape views of the simulation's work fields at table[t] and adds the sensor residual r_t:
// lambda_p += Sample^T r_t, and x1 = tau c^2 lambda_p, x2 = eta c^2 lambda_p at the same points.
void launch_adj_begin(cudaStream_t st, SimDev* d_sims, int* d_t, const int* d_rev, const AdjTapeEntry* table,
                      const float* resid, int npts);
// copy p, S, div of the current state (step t = *d_t - 1) into table[t] (a restored checkpoint, or
// step 0 whose t = 0 override follows its epilogues)
void launch_adj_tape(cudaStream_t st, SimDev* d_sims, const int* d_t, const AdjTapeEntry* table, int stokes, long long N);
// point the tape views of the work fields at table[t] (no step counter change)
void launch_adj_views(cudaStream_t st, SimDev* d_sims, const AdjTapeEntry* table, int t);
void launch_adj_eos(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a, int* d_rev, bool grho);
void launch_adj_src(cudaStream_t st, const SimDev* d_sims, int nsrc, const float* gsig, const int* d_t, double* gc);
void launch_adj_vel(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a);
void launch_adj_sum(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a);
void launch_adj_half_dtor(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a);
void launch_adj_p0(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a, const float* p0s, float* gp);
void launch_adj_store_grad(cudaStream_t st, const double* gc, float* out, long long n);
// density gradient: the t = 0 override's u_a = dtor_a / 2 g_a (g_a = D+_a p0 in ADJ_GP):
// dL/d dtor_a += lambda_u_a g_a / 2
void launch_adj_rho_p0(cudaStream_t st, const SimDev* d_sims, long long N);
// dL/drho0 = the direct terms + staggerDensity^T of dL/d rho_sg_a = -dL/d dtor_a dtor_a^2 / dt
void launch_adj_rho_final(cudaStream_t st, const SimDev* d_sims, long long N, float* out);

}  // namespace kw
