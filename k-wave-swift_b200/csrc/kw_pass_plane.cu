// kw_pass_plane.cu — the first two forward passes of a 3D spectral job in one kernel: the R2C
// along C and the FFT along B of one A-plane, on a thread-block cluster that keeps the plane's
// intermediate half spectrum in its distributed shared memory.
//
// Cluster of NC CTAs per plane (item = simulation, component, plane a). CTA `rank` owns rows
// b in [rank RPC, (rank + 1) RPC), RPC = B / NC:
//   phase 1  each row: load the real row, M-point register transform (kw_fft_reg.cuh, threads of
//            a row on consecutive lanes), Hermitian split into X[0 .. M]; X[0] and X[M] are real,
//            so they share slot 0 as X[0] + i X[M]: a row is exactly M complex values in shared
//            memory.
//   cluster barrier
//   phase 2  CTA `rank` takes the packed columns [rank CPC, (rank + 1) CPC), CPC = M / NC: thread t
//            of column line l gathers rows t + T r from the owning CTAs' shared memory (distributed
//            shared memory, 128-byte runs of consecutive columns), runs the B-point transform and
//            stores rows of consecutive columns to the spectrum [A][B][Cp]. The packed column 0
//            holds two real columns: Z = FFT(x_0 + i x_M) gives X_0(k) = (Z(k) + conj Z(-k)) / 2
//            and X_M(k) = (Z(k) - conj Z(-k)) / 2i.
//   cluster barrier (no CTA leaves while its rows may still be read)
// The result equals the R2C pass followed by the forward column pass along B; the spectrum
// makes one HBM round trip fewer.
#include <cooperative_groups.h>

#include "kw_fft_reg.cuh"
#include "kw_pass_common.cuh"

namespace cg = cooperative_groups;

namespace kw {

template <int M, int NB, int NC>
struct PlaneCfg {
    using PR = RegPlan<M, reg_r1(M)>;     // row transform
    using LR = RowLayout<PR, M>;
    using PC = RegPlan<NB, reg_r1(NB)>;   // column transform
    using LC = ColLayout<PC, NB>;
    static constexpr int RPC = NB / NC;   // rows per CTA
    static constexpr int CPC = M / NC;    // packed columns per CTA
    static constexpr int LDR = M + 1;     // row stride in shared memory (complex values)
    static constexpr int ROWS = RPC * LDR * 8;
    static constexpr int EXCH = (LR::SLOTS > LC::SLOTS ? LR::SLOTS : LC::SLOTS) * 8;
    static constexpr int SMEM = ROWS + EXCH;
    static_assert(NB % NC == 0 && M % NC == 0, "plane split");
    static_assert(ROWS % 16 == 0, "alignment");
};

template <int M, int NB, int NC>
__global__ void __cluster_dims__(NC, 1, 1) __launch_bounds__(256, 2)
    k_plane_r2c(const SimDev* __restrict__ sims, const int* __restrict__ d_t, const BlockWork* __restrict__ map,
                int nmap, RowR2CJob job) {
    using Cfg = PlaneCfg<M, NB, NC>;
    extern __shared__ __align__(16) unsigned char smem[];
    float2* rows = reinterpret_cast<float2*>(smem);
    float2* sh = reinterpret_cast<float2*>(smem + Cfg::ROWS);
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int item = blockIdx.x / NC;
    // every CTA of a cluster takes the same exits (the grid is nmap * NC, the gate is per item)
    if (item >= nmap) return;
    const BlockWork bw = map[item];
    const SimDev& S = sims[bw.sim];
    if (!gate_open(S, job.gate, bw.comp, *d_t)) return;
    const int a = bw.tile;

    // ---- phase 1: R2C of this CTA's rows into shared memory ----
    {
        using P = typename Cfg::PR;
        using Lay = typename Cfg::LR;
        constexpr int R1 = P::R1, T = P::T, TW = P::LINES;
        const int t = threadIdx.x % T, l = threadIdx.x / T;
        const float* f = field_ptr(S, job.in_field, bw.comp) + (long long)a * NB * (2 * M);
        const float2* __restrict__ tw = S.row_tw;
        auto bin = [&](int k, float2 zk, float2 zm) {
            const float2 E = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
            const float2 D = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y + zm.y));
            const float2 O = make_float2(D.y, -D.x);   // -i D
            return cadd(E, cmul(O, __ldg(tw + k)));
        };
#pragma unroll 1
        for (int r0 = 0; r0 < Cfg::RPC; r0 += TW) {
            const int lr = r0 + l;
            const bool ok = lr < Cfg::RPC;
            const float2* in = reinterpret_cast<const float2*>(f + (long long)(rank * Cfg::RPC + (ok ? lr : 0)) * (2 * M));
            float2 v[R1];
#pragma unroll
            for (int r = 0; r < R1; ++r) v[r] = ok ? in[t + T * r] : make_float2(0.f, 0.f);
            FftReg<M, P, false, Lay>::run(v, sh, t, l, S.plan_row.twn);
            // the split needs Z[M - k], held by another thread of the row
#pragma unroll
            for (int m = 0; m < R1; ++m) sh[Lay::at(t + T * m, l)] = v[m];
            __syncthreads();
            if (ok) {
                float2* out = rows + lr * Cfg::LDR;
#pragma unroll
                for (int m = 0; m < R1; ++m) {
                    const int k = t + T * m;
                    const float2 X = bin(k, v[m], sh[Lay::at(k == 0 ? 0 : M - k, l)]);
                    out[k] = k == 0 ? make_float2(X.x, bin(M, v[0], v[0]).x) : X;   // slot 0: X[0] + i X[M]
                }
            }
            __syncthreads();   // the exchange buffer is reused by the next round
        }
    }
    cluster.sync();

    // ---- phase 2: FFT along B of this CTA's packed columns, gathered across the cluster ----
    {
        using P = typename Cfg::PC;
        using Lay = typename Cfg::LC;
        constexpr int R1 = P::R1, T = P::T, TW = P::LINES;
        const int l = threadIdx.x % TW, t = threadIdx.x / TW;
        float2* out = S.spec[job.spec_out + bw.comp] + (long long)a * NB * S.Cp;
        const float2* __restrict__ twn = S.plan_b.twn;
#pragma unroll 1
        for (int c0 = 0; c0 < Cfg::CPC; c0 += TW) {
            const bool ok = c0 + l < Cfg::CPC;
            const int kc = rank * Cfg::CPC + c0 + (ok ? l : 0);
            float2 v[R1];
#pragma unroll
            for (int r = 0; r < R1; ++r) {
                const int b = t + T * r;
                const int owner = b / Cfg::RPC;
                const float2* src = cluster.map_shared_rank(rows, owner);
                v[r] = ok ? src[(b - owner * Cfg::RPC) * Cfg::LDR + kc] : make_float2(0.f, 0.f);
            }
            FftReg<NB, P, false, Lay>::run(v, sh, t, l, twn);
            const bool packed = rank == 0 && c0 == 0;   // uniform over the CTA
            if (packed) {
                // unpack line 0: X_0(k) = (Z(k) + conj Z(-k)) / 2, X_M(k) = (Z(k) - conj Z(-k)) / 2i
                if (l == 0) {
#pragma unroll
                    for (int m = 0; m < R1; ++m) sh[t + T * m] = v[m];
                }
                __syncthreads();
                if (l == 0) {
#pragma unroll
                    for (int m = 0; m < R1; ++m) {
                        const int k = t + T * m;
                        const float2 z = v[m], zm = sh[k == 0 ? 0 : NB - k];
                        const float2 x0 = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
                        const float2 dd = make_float2(z.x - zm.x, z.y + zm.y);
                        const float2 xm = make_float2(0.5f * dd.y, -0.5f * dd.x);
                        out[(long long)k * S.Cp] = x0;
                        out[(long long)k * S.Cp + M] = xm;
                    }
                }
                __syncthreads();
            }
            if (ok && !(packed && l == 0)) {
#pragma unroll
                for (int m = 0; m < R1; ++m) out[(long long)(t + T * m) * S.Cp + kc] = v[m];
            }
        }
    }
    cluster.sync();
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
// (M = C / 2, B, cluster size): the shared-memory rows of a CTA stay under ~80 KB
#define KW_PLANE_CONFIGS(X) X(16, 32, 1) X(32, 64, 1) X(24, 48, 1) X(48, 48, 1) X(64, 64, 2) X(64, 128, 2) \
    X(128, 128, 4) X(128, 256, 4) X(96, 192, 2) X(192, 384, 8)

int plane_cluster(int M, int NB) {
#define KW_MATCH(m, nb, nc) \
    if (M == m && NB == nb) return nc;
    KW_PLANE_CONFIGS(KW_MATCH)
#undef KW_MATCH
    return 0;
}

void init_plane_attributes(int optin) {
    (void)optin;
#define KW_SET(m, nb, nc)                                                                                     \
    cudaFuncSetAttribute((const void*)k_plane_r2c<m, nb, nc>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                         PlaneCfg<m, nb, nc>::SMEM);
    KW_PLANE_CONFIGS(KW_SET)
#undef KW_SET
}

void launch_plane_r2c(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                      const RowR2CJob& job, int M, int NB) {
    if (nmap <= 0) return;
#define KW_CASE(m, nb, nc)                                                                                      \
    if (M == m && NB == nb) {                                                                                   \
        k_plane_r2c<m, nb, nc><<<nmap * nc, 256, PlaneCfg<m, nb, nc>::SMEM, st>>>(d_sims, d_t, map, nmap, job); \
        return;                                                                                                 \
    }
    KW_PLANE_CONFIGS(KW_CASE)
#undef KW_CASE
}

}  // namespace kw
