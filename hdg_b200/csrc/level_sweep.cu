// level_sweep.cu -- BILU(0) application (kernel/applyBILU0.m:10-48) as ONE launch per apply.
//
// A sequential elimination order such as the minimum-discarded-fill order of
// kernel/computeMDFordering.m has long dependency chains: on the 2D NS p = 3 mesh of 49,408
// faces the level schedule has 1,100 levels of 45 rows on average.  One launch per level and
// sweep costs ~13 us of launch gap and dependent index loads per level.  Here a single thread-
// block cluster (CS CTAs, co-scheduled by the hardware) walks all levels of the forward and
// the backward sweep; the levels are separated by the hardware cluster barrier, so no flag is
// polled and no wait can hang.  Every row's dependencies are pre-flattened on the host into one
// fixed-width record (row, diagonal block, (block, column) pairs of the earlier and of the later
// neighbours), so a thread reaches its data with one load instead of a chain of index loads,
// and the record and matrix values of the next level (which do not depend on this level's
// results) are loaded between the barrier's arrive and its wait.
//
// Work split inside a level: rows s = 0..nr-1 of the level go to CTA s % CS; inside a CTA a
// pass covers NT / BS rows with one thread per row component r.  The forward sweep computes
//   y_i[r] = x_i[r] - sum_j L_ij[r, :] y_j        (rows j eliminated before i)
// and the backward sweep
//   t_i[r] = y_i[r] - sum_j U_ij[r, :] v_j        (rows j eliminated after i)
//   v_i[r] = sum_c inv(U_ii)[r, c] t_i[c]         (diagonal blocks are stored inverted)
// in the operation order of the per-level kernels.  Values written in one level are read in a
// later one by other CTAs: the writes are followed by a GPU-scope fence before the barrier's
// arrive, the wait has acquire semantics, and those reads go through L2 (ld.global.cg).
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include "hdgx_common.cuh"

namespace cg = cooperative_groups;

namespace hdgx {

__device__ __forceinline__ void cluster_arrive_relaxed() {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait_acquire() {
    asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
// the 16-byte aligned interior of [p, p + bytes) into L2 (a bulk prefetch needs aligned ends)
__device__ __forceinline__ void bulk_prefetch_l2(const void *p, unsigned bytes) {
    const unsigned long long a0 = ((unsigned long long)p + 15) & ~15ull;
    const unsigned long long a1 = ((unsigned long long)p + bytes) & ~15ull;
    if (a1 > a0) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a0), "r"((unsigned)(a1 - a0)) : "memory");
}

// One row component's record and (PL) matrix values, loadable ahead of the level that uses them.
// MT is the storage type of the factors (double, or float for the mixed-precision preconditioner:
// the values are widened on use and every sum runs in FP64).
template <int BS, int MAXD, bool PL, bool DIAG, class MT>
struct RowPrefetch {
    int i, k0;
    int k[MAXD], j[MAXD];
    MT lv[PL ? MAXD * BS : 1];
    MT dv[(PL && DIAG) ? BS : 1];

    // slot record R (NULL: inactive); OFF = 0 for the earlier neighbours, 2 * MAXD for the later
    template <int OFF>
    __device__ __forceinline__ void load(const int *R, const MT *__restrict__ Mg, int r) {
        if (!R) { i = -1; return; }
        i = __ldg(R);
        k0 = __ldg(R + 1);
#pragma unroll
        for (int d = 0; d < MAXD; d++) { k[d] = __ldg(R + 2 + OFF + 2 * d); j[d] = __ldg(R + 3 + OFF + 2 * d); }
        if constexpr (PL) {
#pragma unroll
            for (int d = 0; d < MAXD; d++) {
                if (k[d] >= 0) {
                    const MT *B = Mg + (size_t)BS * BS * k[d] + r;
#pragma unroll
                    for (int c = 0; c < BS; c++) lv[d * BS + c] = __ldg(B + BS * c);
                } else {
#pragma unroll
                    for (int c = 0; c < BS; c++) lv[d * BS + c] = MT(0);     // padded slot: contributes 0
                }
            }
            if constexpr (DIAG) {
                const MT *D = Mg + (size_t)BS * BS * k0 + r;
#pragma unroll
                for (int c = 0; c < BS; c++) dv[c] = __ldg(D + BS * c);
            }
        }
    }

    // acc - sum_d B_d[r, :] in_{j_d}
    __device__ __forceinline__ double reduce(double acc, const MT *__restrict__ Mg, const double *in, int r) const {
        if constexpr (PL) {
            // every neighbour's values are loaded before the first multiply-add, so their L2
            // round trips overlap; padded slots (k < 0) contribute exact zeros
            double ov[MAXD][BS];
#pragma unroll
            for (int d = 0; d < MAXD; d++) {
                const bool live = k[d] >= 0;
                const double *oj = in + (size_t)BS * (live ? j[d] : 0);
#pragma unroll
                for (int c = 0; c < BS; c++) ov[d][c] = live ? __ldcg(oj + c) : 0.0;
            }
#pragma unroll
            for (int d = 0; d < MAXD; d++)
#pragma unroll
                for (int c = 0; c < BS; c++) acc -= (double)lv[d * BS + c] * ov[d][c];
            return acc;
        } else {
#pragma unroll
            for (int d = 0; d < MAXD; d++) {
                if (k[d] < 0) break;
                const double *oj = in + (size_t)BS * j[d];
                double ov[BS];
#pragma unroll
                for (int c = 0; c < BS; c++) ov[c] = __ldcg(oj + c);
                const MT *B = Mg + (size_t)BS * BS * k[d] + r;
                double bv[BS];
#pragma unroll
                for (int c = 0; c < BS; c++) bv[c] = (double)__ldg(B + BS * c);
#pragma unroll
                for (int c = 0; c < BS; c++) acc -= bv[c] * ov[c];
            }
            return acc;
        }
    }

    // sum_c inv(U_ii)[r, c] t[c]
    __device__ __forceinline__ double diag(const MT *__restrict__ Mg, const double *t, int r) const {
        double o = 0.0;
        if constexpr (PL && DIAG) {
#pragma unroll
            for (int c = 0; c < BS; c++) o += (double)dv[c] * t[c];
        } else {
            const MT *D = Mg + (size_t)BS * BS * k0 + r;
#pragma unroll
            for (int c = 0; c < BS; c++) o += (double)__ldg(D + BS * c) * t[c];
        }
        return o;
    }
};

template <int BS, int MAXD, int CS, int NT, class MT>
__global__ void __cluster_dims__(CS, 1, 1) __launch_bounds__(NT)
    bilu0_level_sweep_kernel(int nlev, const int *__restrict__ plan, const MT *__restrict__ Mg,
                             const double *__restrict__ x, double *y, double *v) {
    constexpr int RPP = NT / BS;                        // rows per pass per CTA
    constexpr int RW = 2 + 4 * MAXD;                    // record width (ints)
    constexpr bool PLF = MAXD * BS <= 64;               // forward: L values prefetched
    constexpr bool PLB = (MAXD + 1) * BS <= 80;         // backward: U and inv(D) values prefetched
    extern __shared__ int lp[];                         // level offsets [nlev + 1]
    __shared__ double tsh[RPP * BS];
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int *rec = plan + nlev + 1;
    const int m = threadIdx.x / BS, r = threadIdx.x - (threadIdx.x / BS) * BS;
    for (int t = threadIdx.x; t <= nlev; t += NT) lp[t] = __ldg(plan + t);
    __syncthreads();
    auto slot_rec = [&](int lev) -> const int * {      // this thread's first-pass record, or NULL
        const int q0 = lp[lev], nr = lp[lev + 1] - q0, s = rank + CS * m;
        return (m < RPP && s < nr) ? rec + (size_t)(q0 + s) * RW : nullptr;
    };
    // L2 pipeline for the first pass of later levels (the factors are read once per apply and
    // do not stay in L2 between applies): the records of level lev + DR are prefetched to L2;
    // one block index per thread (component r < NK of the row: a neighbour block, in the
    // backward sweep r = 0 the diagonal block) is loaded DK levels ahead and its block
    // prefetched to L2 one level later, so the register prefetch of the next level hits L2.
    constexpr int DR = 7, DK = 4;
    auto prefetch_rec = [&](int lev) {
        if (r == 0 && lev >= 0 && lev < nlev) {
            const int *R = slot_rec(lev);
            if (R) { prefetch_l2(R); prefetch_l2(R + RW - 1); }
        }
    };
    // the block index component r prefetches at level lev (-1: none); BWD: backward-sweep blocks
    auto block_of = [&](int lev, bool bwd) -> int {
        if (lev < 0 || lev >= nlev) return -1;
        const int *R = slot_rec(lev);
        if (!R) return -1;
        if (!bwd) return r < MAXD ? __ldcg(R + 2 + 2 * r) : -1;
        return r == 0 ? __ldcg(R + 1) : (r <= MAXD ? __ldcg(R + 2 + 2 * MAXD + 2 * (r - 1)) : -1);
    };
    auto prefetch_block = [&](int k) {
        if (k >= 0) bulk_prefetch_l2(Mg + (size_t)BS * BS * k, (unsigned)(sizeof(MT) * BS * BS));
    };

    // forward sweep: y_i = x_i - sum_{j before i} L_ij y_j, levels in elimination order
    {
        for (int l = 0; l < DR; l++) prefetch_rec(l);
        int pk = block_of(DK - 1, false);
        RowPrefetch<BS, MAXD, PLF, false, MT> pf;
        pf.template load<0>(slot_rec(0), Mg, r);
        double xv = pf.i >= 0 ? __ldg(x + (size_t)BS * pf.i + r) : 0.0;
        for (int lev = 0; lev < nlev; lev++) {
            const int q0 = lp[lev], nr = lp[lev + 1] - q0;
            if (pf.i >= 0) y[(size_t)BS * pf.i + r] = pf.reduce(xv, Mg, y, r);
            for (int base = CS * RPP; base < nr; base += CS * RPP) {
                const int s = base + rank + CS * m;
                if (m < RPP && s < nr) {
                    RowPrefetch<BS, MAXD, false, false, MT> row;
                    row.template load<0>(rec + (size_t)(q0 + s) * RW, Mg, r);
                    y[(size_t)BS * row.i + r] = row.reduce(__ldg(x + (size_t)BS * row.i + r), Mg, y, r);
                }
            }
            __threadfence();
            cluster_arrive_relaxed();
            if (lev + 1 < nlev) {
                pf.template load<0>(slot_rec(lev + 1), Mg, r);
                xv = pf.i >= 0 ? __ldg(x + (size_t)BS * pf.i + r) : 0.0;
            }
            prefetch_block(pk);                         // level lev + DK - 1
            pk = block_of(lev + DK, false);
            prefetch_rec(lev + DR);
            cluster_wait_acquire();
        }
    }
    // backward sweep: v_i = inv(U_ii) (y_i - sum_{j after i} U_ij v_j), levels in reverse order
    {
        for (int l = 0; l < DR; l++) prefetch_rec(nlev - 1 - l);
        int pk = block_of(nlev - DK, true);
        RowPrefetch<BS, MAXD, PLB, true, MT> pf;
        pf.template load<2 * MAXD>(slot_rec(nlev - 1), Mg, r);
        for (int lev = nlev - 1; lev >= 0; lev--) {
            const int q0 = lp[lev], nr = lp[lev + 1] - q0;
            // pass 0 (prefetched); y_i[r] was written by this same thread in the forward sweep
            if (pf.i >= 0) tsh[m * BS + r] = pf.reduce(__ldcg(y + (size_t)BS * pf.i + r), Mg, v, r);
            __syncthreads();
            if (pf.i >= 0) v[(size_t)BS * pf.i + r] = pf.diag(Mg, tsh + m * BS, r);
            if (nr > CS * RPP) __syncthreads();      // tsh is rewritten by the next pass (else the
                                                     // cluster barrier below orders its reuse)
            for (int base = CS * RPP; base < nr; base += CS * RPP) {    // trip count is uniform in the CTA
                const int s = base + rank + CS * m;
                const bool act = m < RPP && s < nr;
                RowPrefetch<BS, MAXD, false, true, MT> row;
                row.template load<2 * MAXD>(act ? rec + (size_t)(q0 + s) * RW : nullptr, Mg, r);
                if (act) tsh[m * BS + r] = row.reduce(__ldcg(y + (size_t)BS * row.i + r), Mg, v, r);
                __syncthreads();
                if (act) v[(size_t)BS * row.i + r] = row.diag(Mg, tsh + m * BS, r);
                __syncthreads();
            }
            __threadfence();
            cluster_arrive_relaxed();
            if (lev > 0) pf.template load<2 * MAXD>(slot_rec(lev - 1), Mg, r);
            prefetch_block(pk);                         // level lev - DK + 1
            pk = block_of(lev - DK, true);
            prefetch_rec(lev - DR);
            cluster_wait_acquire();
        }
    }
}

constexpr int kSweepCS = 8;     // CTAs in the cluster (portable maximum)
constexpr int kSweepNT = 256;

// 0 launched, 1 not possible (caller falls back), 2 the device cannot place such a cluster
template <int BS, int MAXD, int CS, int NT, class MT>
static int launch_cluster(int nlev, const int *plan, const MT *Mg, const double *x, double *y, double *v,
                          size_t smem, cudaStream_t st) {
    auto kern = bilu0_level_sweep_kernel<BS, MAXD, CS, NT, MT>;
    if (smem > 40 * 1024 && allow_dynamic_smem((const void *)kern, smem) != cudaSuccess) return 1;
    if (CS > 8) {
        if (cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
            cudaGetLastError();
            return 2;
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(CS);
        cfg.blockDim = dim3(NT);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = st;
        int ncl = 0;
        if (cudaOccupancyMaxActiveClusters(&ncl, (const void *)kern, &cfg) != cudaSuccess || ncl < 1) {
            cudaGetLastError();
            return 2;
        }
    }
    kern<<<CS, NT, smem, st>>>(nlev, plan, Mg, x, y, v);
    return 0;
}

// Large blocks (bs >= 20: 3D, or 2D p = 4) run CTAs of 512 threads (fewer passes per level).
// When a level moves more matrix than 8 SMs stream in the time of a level (kWideLevelBytes of
// factors per level on average) the cluster has 16 CTAs (a non-portable size) when the device
// can place one, else 8.  (3D Euler p = 2, 399,360 faces, 12 MB per level: 69.5 ms per apply
// with 8 CTAs of 256, 57.9 ms with 8 of 512, 37.2 ms with 16 of 512.)  Small systems stay on 8:
// a 16-CTA cluster needs 16 free SMs of one GPC, which concurrent solves rarely leave (64 queued
// serving requests: 32 solves/s with 16-CTA clusters for their bs = 20 systems, 74 with 8).
constexpr size_t kWideLevelBytes = 4u << 20;
template <int BS, int MAXD, class MT>
static int launch_level_sweep(int nlev, long long nnzb, const int *plan, const MT *Mg, const double *x, double *y,
                              double *v, cudaStream_t st) {
    const size_t smem = sizeof(int) * ((size_t)nlev + 1);
    if (smem > 160 * 1024) return 1;                    // very long schedules: per-level launches
    if constexpr (BS >= 20) {
        const size_t level_bytes = sizeof(MT) * BS * BS * (size_t)nnzb / (size_t)nlev;
        if (level_bytes >= kWideLevelBytes) {
            const int rc = launch_cluster<BS, MAXD, 16, 512, MT>(nlev, plan, Mg, x, y, v, smem, st);
            if (rc != 2) return rc;
        }
        return launch_cluster<BS, MAXD, 8, 512, MT>(nlev, plan, Mg, x, y, v, smem, st) == 0 ? 0 : 1;
    } else {
        return launch_cluster<BS, MAXD, kSweepCS, kSweepNT, MT>(nlev, plan, Mg, x, y, v, smem, st) == 0 ? 0 : 1;
    }
}

// 0 when launched, 1 when there is no plan or no specialisation for it (the caller falls back)
template <class MT>
static int level_sweep_apply_t(const hdgx_bsr *A, const MT *Mg, const double *x, double *y, double *v, cudaStream_t st) {
    if (!A->sweep_plan || A->ncolors < 1) return 1;
    const int md = A->sweep_maxd;
    if (md != 4 && md != 6) return 1;
    switch (A->bs) {
#define HDGX_LS(B)                                                                                \
    case B:                                                                                       \
        return md == 4 ? launch_level_sweep<B, 4, MT>(A->ncolors, A->nnzb, A->sweep_plan, Mg, x, y, v, st)    \
                       : launch_level_sweep<B, 6, MT>(A->ncolors, A->nnzb, A->sweep_plan, Mg, x, y, v, st);
        HDGX_LS(8) HDGX_LS(12) HDGX_LS(15) HDGX_LS(16) HDGX_LS(20) HDGX_LS(30)
#undef HDGX_LS
        default: return 1;
    }
}

int level_sweep_apply(const hdgx_bsr *A, const double *Mg, const double *x, double *y, double *v, cudaStream_t st) {
    return level_sweep_apply_t<double>(A, Mg, x, y, v, st);
}
// The same sweeps with the factors stored in FP32 (the mixed-precision preconditioner)
int level_sweep_apply_f32(const hdgx_bsr *A, const float *Mg, const double *x, double *y, double *v, cudaStream_t st) {
    return level_sweep_apply_t<float>(A, Mg, x, y, v, st);
}

}  // namespace hdgx
