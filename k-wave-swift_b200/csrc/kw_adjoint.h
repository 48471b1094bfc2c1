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
    ADJ_X1 = 13,      // tau c^2 lambda_p      } job A1 inputs
    ADJ_DIVT = 14,    // div(t) from the tape  }
    ADJ_A1 = 15,      // A1(tau c^2 lambda_p)  } job A1 outputs
    ADJ_Q1 = 16,      // A1(div(t))            }
    ADJ_X2 = 17,      // eta c^2 lambda_p      } job A2 inputs
    ADJ_ST = 18,      // S(t) from the tape    }
    ADJ_A2 = 19,      // A2(eta c^2 lambda_p)  } job A2 outputs
    ADJ_Q2 = 20,      // A2(S(t))              }
    ADJ_SIG = 21,     // sum_a L_a / dx_a
    ADJ_GSIG = 22,    // G(sigma)
    ADJ_UT = 23,      // u_a(t) from the tape, 3
    ADJ_DD = 26,      // D-_a u_a(t), 3
    ADJ_PT = 29,      // p(t) from the tape
    ADJ_SPREV = 30,   // S(t-1)
    ADJ_COUNT = 31
};
static_assert(ADJ_COUNT <= kAdjFields, "adjoint fields");

// device pointers of one reverse step
struct AdjStepArgs {
    const float* pt;
    const float* st;
    const float* sprev;
    const float* divt;
    const float* a1;
    const float* a2;
    const float* q1;
    const float* q2;
    const float* dd[kMaxComp];
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
void launch_adj_residual(cudaStream_t st, const SimDev* d_sims, int npts, const float* resid, int t, float* lam_p);
void launch_adj_pre(cudaStream_t st, const SimDev* d_sims, long long N, const float* lam_p, float* x1, float* x2);
void launch_adj_eos(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a);
void launch_adj_src(cudaStream_t st, const SimDev* d_sims, int nsrc, const float* gsig, int t, double* gc);
void launch_adj_vel(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a);
void launch_adj_sum(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a);
void launch_adj_half_dtor(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a);
void launch_adj_p0(cudaStream_t st, const SimDev* d_sims, long long N, const AdjStepArgs& a, const float* p0s, float* gp);
void launch_adj_store_grad(cudaStream_t st, const double* gc, float* out, long long n);

}  // namespace kw
