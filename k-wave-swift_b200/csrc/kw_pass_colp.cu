// kw_pass_colp.cu — warp-specialised, TMA-fed in-place column pass for the register-plan lengths.
//
// A persistent CTA of 9 warps walks its share of the launch's tiles. Warp 8 (one lane) is the
// producer: it loads each tile — colr_lines(N) columns by the N rows of the pass axis — with one
// TMA tensor copy into a ring of NS shared-memory stages, completing on the stage's `full` mbarrier. Warps 0-7 are the consumers:
// they wait for the stage, pick up their register values x[t + T r] of line l (consecutive lanes
// read consecutive columns), release the stage on its `empty` mbarrier (one arrival per warp) and
// run the register-resident transform of kw_fft_reg.cuh, synchronising among themselves with named
// barrier 1. Results go straight from registers to HBM. The ring keeps up to NS tiles of loads in
// flight per SM while the consumers compute, so the pass streams at HBM speed instead of waiting
// on each tile's loads.
//
// The in-place forward / inverse passes (COL_FWD / COL_INV) use it; the operator pass is
// kw_pass_colop.cu. Every wait is bounded (kw_async.cuh).
#include "kw_async.cuh"
#include "kw_fft_reg.cuh"
#include "kw_pass_common.cuh"

namespace kw {

template <int N>
struct ColpCfg {
    using P = RegPlan<N, reg_r1(N)>;
    static constexpr int TW = P::LINES;
    static constexpr int STAGE = N * TW * 8;   // one tile: TW columns by N rows
    static constexpr int EXCH = ColLayout<P, N>::SLOTS * 8;
    // two resident CTAs per SM, so that one's transform overlaps the other's
    static constexpr int MINB = 2;
    static constexpr int BUDGET = (224 * 1024) / MINB;   // shared memory of one CTA
    static constexpr int NS_FIT = (BUDGET - EXCH - 256) / STAGE;
    static constexpr int NS = NS_FIT > 6 ? 6 : NS_FIT;
    static constexpr int BAR_OFF = NS * STAGE + EXCH;
    static constexpr int SMEM = BAR_OFF + 2 * NS * 8;
    static_assert(NS >= 2, "at least two stages");
    static_assert(STAGE % 128 == 0 && EXCH % 16 == 0, "stage alignment");
};

template <int N, bool INV>
__global__ void __launch_bounds__(288, ColpCfg<N>::MINB) k_colp(const SimDev* __restrict__ sims, const int* __restrict__ d_t,
                                                                const BlockWork* __restrict__ map, int nmap, ColJob job,
                                                                int* __restrict__ err) {
    pdl_enter();
    using Cfg = ColpCfg<N>;
    using P = typename Cfg::P;
    using Lay = ColLayout<P, N>;
    constexpr int R1 = P::R1, T = P::T, TW = Cfg::TW, NS = Cfg::NS;
    extern __shared__ __align__(128) unsigned char smem[];
    float2* sh = reinterpret_cast<float2*>(smem + NS * Cfg::STAGE);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + Cfg::BAR_OFF);
    uint64_t* empty = full + NS;
    __shared__ volatile int abort;   // set by the consumers when one of their waits ran out
    if (threadIdx.x == 0) {
        abort = 0;
        for (int s = 0; s < NS; ++s) {
            mbar_init(full + s, 1);
            mbar_init(empty + s, 8);
        }
        fence_barrier_init();
    }
    __syncthreads();
    const int tstep = *d_t;
    const bool axisA = job.layout_axis == 0;

    if (threadIdx.x >= 256) {
        // ---------------- producer ----------------
        if (threadIdx.x != 256) return;
        int k = 0;
        bool withheld = false;   // test hook (SimDev::test_stall): the first tile's copy was not issued
        for (int idx = blockIdx.x; idx < nmap; idx += gridDim.x) {
            const BlockWork bw = map[idx];
            const SimDev& S = sims[bw.sim];
            if (!gate_open(S, job.gate, bw.comp, tstep)) continue;
            const int s = k % NS;
            if (k >= NS && !mbar_wait_or_abort(empty + s, ((k / NS) & 1) ^ 1, err, KE_TIMEOUT_EMPTY, &abort)) break;
            const int inner = axisA ? S.B * S.Cp : S.Cp;
            const int nch = (inner + TW - 1) / TW;
            const int o = bw.tile / nch;
            const int c0 = (bw.tile - o * nch) * TW;
            const int comp_in = job.fanout ? 0 : bw.comp;
            unsigned char* st = smem + s * Cfg::STAGE;
            if (S.test_stall && k == 0) {
                withheld = true;   // its consumers' bounded wait runs out: nothing completes the barrier
            } else {
                mbar_arrive_expect_tx(full + s, Cfg::STAGE);
                const CUtensorMap* tm = S.tmaps + tmap_spec(job.spec_in + comp_in, job.layout_axis);
                if (axisA) tma_load_2d(st, tm, c0, 0, full + s);
                else tma_load_3d(st, tm, c0, 0, o, full + s);
                // the tile job.tma_ahead of this CTA's tiles on, into L2 (beyond the ring's reach)
                const int pidx = idx + job.tma_ahead * gridDim.x;
                if (job.tma_ahead > 0 && pidx < nmap) {
                    const BlockWork pw = map[pidx];
                    const SimDev& P2 = sims[pw.sim];
                    const int pinner = axisA ? P2.B * P2.Cp : P2.Cp;
                    const int pnch = (pinner + TW - 1) / TW;
                    const int po = pw.tile / pnch;
                    const int pc0 = (pw.tile - po * pnch) * TW;
                    const CUtensorMap* ptm = P2.tmaps + tmap_spec(job.spec_in + (job.fanout ? 0 : pw.comp), job.layout_axis);
                    if (axisA) tma_prefetch_2d(ptm, pc0, 0);
                    else tma_prefetch_3d(ptm, pc0, 0, po);
                }
            }
            ++k;
        }
        // every issued copy must have landed before this CTA's shared memory is released
        for (int j = k > NS ? k - NS : 0; j < k; ++j)
            if (!(withheld && j == 0)) mbar_wait(full + j % NS, (j / NS) & 1, err, KE_TIMEOUT_DRAIN);
        return;
    }

    // ---------------- consumers ----------------
    const int l = threadIdx.x % TW;
    const int t = threadIdx.x / TW;
    const int lane = threadIdx.x & 31;
    int k = 0;
    for (int idx = blockIdx.x; idx < nmap; idx += gridDim.x) {
        const BlockWork bw = map[idx];
        const SimDev& S = sims[bw.sim];
        if (!gate_open(S, job.gate, bw.comp, tstep)) continue;
        const int s = k % NS;
        // (the limit is the simulation's: a test shortens it to make this wait run out; the
        // producer's waits keep the default, so it still drains its copies before exiting)
        const bool ok = mbar_wait(full + s, (k / NS) & 1, err, KE_TIMEOUT_FULL, S.wait_cycles);
        // all consumers agree before anyone touches the stage or a barrier
        int all_ok;
        asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.and.pred q, 1, 256, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
                     : "=r"(all_ok) : "r"((unsigned)ok) : "memory");
        if (!all_ok) {
            if (threadIdx.x == 0) abort = 1;
            return;
        }
        const float2* tile = reinterpret_cast<const float2*>(smem + s * Cfg::STAGE);

        const int inner = axisA ? S.B * S.Cp : S.Cp;
        const int nch = (inner + TW - 1) / TW;
        const int o = bw.tile / nch;
        const int c = (bw.tile - o * nch) * TW + l;
        const int kc = axisA ? c % S.Cp : c;
        // padding bins (kc >= Ch) stay zero: they are read (as part of the tile) but never written
        const bool col_ok = c < inner && kc < S.Ch;
        const long long base = (long long)o * N * inner + c;
        const float2* __restrict__ twn = axisA ? S.plan_a.twn : S.plan_b.twn;
        const int comp_in = job.fanout ? 0 : bw.comp;

        float2 v[R1];
#pragma unroll
        for (int r = 0; r < R1; ++r) v[r] = tile[(t + T * r) * TW + l];

        __syncwarp();
        if (lane == 0) mbar_arrive(empty + s);
        FftReg<N, P, INV, Lay, ConsumerSync>::run(v, sh, t, l, twn);
        float2* out = S.spec[job.spec_in + comp_in] + base;
        if (col_ok) {
#pragma unroll
            for (int m = 0; m < R1; ++m) out[(long long)(t + T * m) * inner] = v[m];
        }
        ++k;
    }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
template <int N, bool INV>
static void colp_attr() {
    cudaFuncSetAttribute((const void*)k_colp<N, INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, ColpCfg<N>::SMEM);
}

void init_colp_attributes() {
#define KW_SET(n) colp_attr<n, false>(); colp_attr<n, true>();
    KW_COLP_SIZES(KW_SET)
#undef KW_SET
}

template <int N, bool INV>
static void launch_one(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                       const ColJob& job, int* err) {
    using Cfg = ColpCfg<N>;
    static int grid_cap = 0;
    if (!grid_cap) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_colp<N, INV>, 288, Cfg::SMEM);
        grid_cap = sms * (per_sm > 0 ? per_sm : 1);
    }
    const int grid = nmap < grid_cap ? nmap : grid_cap;
    launch_pdl(k_colp<N, INV>, grid, 288, Cfg::SMEM, st, d_sims, d_t, map, nmap, job, err);
}

template <bool INV>
static void launch_dir(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                       const ColJob& job, int n, int* err) {
    switch (n) {
#define KW_CASE(n) \
    case n: launch_one<n, INV>(st, d_sims, d_t, map, nmap, job, err); break;
        KW_COLP_SIZES(KW_CASE)
#undef KW_CASE
        default: break;
    }
}

void launch_colp(cudaStream_t st, const SimDev* d_sims, const int* d_t, const BlockWork* map, int nmap,
                 const ColJob& job, int n, int* err) {
    if (nmap <= 0) return;
    if (job.mode == COL_INV) launch_dir<true>(st, d_sims, d_t, map, nmap, job, n, err);
    else launch_dir<false>(st, d_sims, d_t, map, nmap, job, n, err);
}

}  // namespace kw
