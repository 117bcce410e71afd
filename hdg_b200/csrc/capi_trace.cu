// capi_trace.cu -- extern "C" entry points of the condensed-system path (include/hdgx.h).
#include <cuda_runtime.h>
#include <math.h>
#include <queue>
#include <utility>
#include <vector>
#include "hdgx_common.cuh"
#include "trace_internal.cuh"

namespace hdgx {
__global__ void gather_uh_kernel(int, int, int, const int *, const double *, double *);
__global__ void assemble_h_kernel(int, int, int, long long, const int *, const int *, const int *, const int *,
                                  const int *, const double *, double *);
__global__ void assemble_r_kernel(int, int, int, int, const int *, const int *, const int *, const double *, double *);
__global__ void bsr_matvec_kernel(int, int, const long long *, const int *, const double *, const double *, double *);
template <int NT>
__global__ void bilu0_color_kernel(int, const int *, int, const long long *, const int *, const int *, double *, int *);
__global__ void bilu0_fwd_kernel(int, const int *, int, const long long *, const int *, const int *, const double *,
                                 const double *, double *);
__global__ void bilu0_bwd_kernel(int, const int *, int, const long long *, const int *, const int *, const double *,
                                 const double *, double *);
template <int NT>
__global__ void block_norms_kernel(int, int, const long long *, const double *, double *);
template <int NT>
__global__ void bilu0_sched_factor_kernel(int, int, const int *, const long long *, const int *, const int *, double *,
                                          int *, int *);
__global__ void bilu0_sched_sweep_kernel(int, int, int, const int *, const long long *, const int *, const int *,
                                         const double *, const double *, double *, int *);
__global__ void sched_begin_kernel(int *);
__global__ void backsub_kernel(int, int, int, int, const int *, const double *, const double *, const double *, double *);

template <int BS>
__global__ void bilu0_fwd_bs_kernel(const int *, int, const long long *, const int *, const int *, const double *,
                                    const double *, double *);
template <int BS>
__global__ void bilu0_bwd_bs_kernel(const int *, int, const long long *, const int *, const int *, const double *,
                                    const double *, double *);
template <int BS>
__global__ void bsr_matvec_bs_kernel(int, const long long *, const int *, const double *, const double *, double *);

// SM count of the current device (cached per device ordinal)
static int sm_count() { return sm_count_of(current_device()); }
static unsigned grid_for(size_t n, int threads) {
    size_t g = (n + threads - 1) / threads;
    size_t cap = (size_t)sm_count() * 8;
    if (g > cap) g = cap;
    return (unsigned)(g < 1 ? 1 : g);
}
// 0, or -1000 - cudaError_t of the last failed call (hdgx_status_str decodes it)
static int launched() {
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : -1000 - (int)e;
}

static size_t bilu_smem(int bs) { return sizeof(double) * (4 * (size_t)bs * bs + 200 + 4 + 1); }

int trace_matvec(const hdgx_bsr *A, const double *Hg, const double *x, double *y, cudaStream_t st) {
    const int threads = 256;
    const unsigned grid = grid_for((size_t)A->nf * 32, threads);
    switch (A->bs) {
#define HDGX_MV(B) case B: bsr_matvec_bs_kernel<B><<<grid, threads, 0, st>>>(A->nf, A->rowpts, A->colind, Hg, x, y); break;
        HDGX_MV(8) HDGX_MV(12) HDGX_MV(15) HDGX_MV(16) HDGX_MV(20) HDGX_MV(30)
#undef HDGX_MV
        default: bsr_matvec_kernel<<<grid, threads, 0, st>>>(A->nf, A->bs, A->rowpts, A->colind, Hg, x, y);
    }
    return launched();
}

// one colour (or level) of the forward / backward sweep, block-size specialised when possible
static void sweep_color(const hdgx_bsr *A, int dir, const int *rows, int nr, const double *Mg, const double *in,
                        double *out, cudaStream_t st) {
    const int threads = 256, warps = threads / 32;
    const unsigned grid = (unsigned)((nr + warps - 1) / warps);
    switch (A->bs) {
#define HDGX_SW(B)                                                                                                   \
    case B:                                                                                                           \
        if (dir == 0) bilu0_fwd_bs_kernel<B><<<grid, threads, 0, st>>>(rows, nr, A->rowpts, A->colind, A->pos, Mg, in, out); \
        else bilu0_bwd_bs_kernel<B><<<grid, threads, 0, st>>>(rows, nr, A->rowpts, A->colind, A->pos, Mg, in, out);          \
        return;
        HDGX_SW(8) HDGX_SW(12) HDGX_SW(15) HDGX_SW(16) HDGX_SW(20) HDGX_SW(30)
#undef HDGX_SW
        default: break;
    }
    if (dir == 0) bilu0_fwd_kernel<<<grid, threads, 0, st>>>(A->bs, rows, nr, A->rowpts, A->colind, A->pos, Mg, in, out);
    else bilu0_bwd_kernel<<<grid, threads, sizeof(double) * warps * A->bs, st>>>(A->bs, rows, nr, A->rowpts, A->colind,
                                                                                  A->pos, Mg, in, out);
}

int level_sweep_apply(const hdgx_bsr *A, const double *Mg, const double *x, double *y, double *v, cudaStream_t st);
int level_sweep_apply_f32(const hdgx_bsr *A, const float *Mg, const double *x, double *y, double *v, cudaStream_t st);

int trace_bilu0_apply_f32(const hdgx_bsr *A, const float *Mg32, const double *x, double *y, double *v,
                          cudaStream_t st) {
    if (!A->sweep_plan || A->ncolors < 1) return -2;
    if (level_sweep_apply_f32(A, Mg32, x, y, v, st) != 0) return -2;
    return launched();
}

__global__ void to_f32_kernel(size_t n, const double *__restrict__ a, float *__restrict__ b) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        b[t] = (float)a[t];
}

static int resident_grid(const void *kern, int threads, size_t smem, int cap) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    int g = sm_count() * (per_sm > 0 ? per_sm : 1);
    return g < cap ? g : cap;
}

int trace_bilu0_apply(const hdgx_bsr *A, const double *Mg, const double *x, double *y, double *v, cudaStream_t st) {
    const int threads = 256, warps = threads / 32;
    if (A->ncolors == 0) {
        if (!A->sched) return -1;
        const size_t smem = sizeof(double) * warps * A->bs;
        const int grid = resident_grid((const void *)bilu0_sched_sweep_kernel, threads, smem, (A->nf + warps - 1) / warps);
        sched_begin_kernel<<<1, 1, 0, st>>>(A->sched);
        bilu0_sched_sweep_kernel<<<grid, threads, smem, st>>>(A->bs, A->nf, 0, A->color_rows, A->rowpts, A->colind,
                                                              A->pos, Mg, x, y, A->sched);
        sched_begin_kernel<<<1, 1, 0, st>>>(A->sched);
        bilu0_sched_sweep_kernel<<<grid, threads, smem, st>>>(A->bs, A->nf, 1, A->color_rows, A->rowpts, A->colind,
                                                              A->pos, Mg, y, v, A->sched);
        return launched();
    }
    (void)warps;
    if (A->sweep_plan && level_sweep_apply(A, Mg, x, y, v, st) == 0) return launched();
    for (int c = 0; c < A->ncolors; c++) {
        const int r0 = A->color_ptr[c], nr = A->color_ptr[c + 1] - r0;
        if (nr > 0) sweep_color(A, 0, A->color_rows + r0, nr, Mg, x, y, st);
    }
    for (int c = A->ncolors - 1; c >= 0; c--) {
        const int r0 = A->color_ptr[c], nr = A->color_ptr[c + 1] - r0;
        if (nr > 0) sweep_color(A, 1, A->color_rows + r0, nr, Mg, y, v, st);
    }
    return launched();
}

__global__ void mgs_coop_kernel(size_t, int, const double *, double *, double *, double *, unsigned *, int *);

// The Arnoldi orthogonalisation of w against V(:, 0:nv) and its normalisation as one cooperative
// launch (mgs_coop_kernel); false when the device cannot hold the grid at once (the caller then
// issues the separate products).  part: 2 * 1024 doubles; bar: 2 unsigned (bar[0] == 0 on entry).
static bool mgs_fused(size_t n, int nv, const double *V, double *w, double *hcol, double *part, unsigned *bar, int *err,
                      cudaStream_t st) {
    unsigned grid = grid_for(n, 256);
    if (grid > 1024) grid = 1024;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)mgs_coop_kernel, 256, 0) != cudaSuccess ||
        (long long)per_sm * sm_count() < (long long)grid) {
        cudaGetLastError();
        return false;
    }
    void *args[] = {&n, &nv, &V, &w, &hcol, &part, &bar, &err};
    if (cudaLaunchCooperativeKernel((const void *)mgs_coop_kernel, dim3(grid), dim3(256), args, 0, st) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

// dot(a,b) -> *out (device); part: scratch of >= 1024 doubles
static void dot(size_t n, const double *a, const double *b, double *out, double *part, int do_sqrt, cudaStream_t st) {
    const int threads = 256;
    unsigned grid = grid_for(n, threads);
    if (grid > 1024) grid = 1024;
    dot_partial_kernel<<<grid, threads, 0, st>>>(n, a, b, part);
    dot_final_kernel<<<1, 256, 0, st>>>((int)grid, part, out, do_sqrt);
}
}  // namespace hdgx

using namespace hdgx;

extern "C" {

int hdgx_gather_uh(int ncu, int ndf, int ne, const int *elcon, const double *UH, double *UHe, hdgx_stream_t stream) {
    if (ne < 0 || ncu < 1 || ndf < 1) return -1;
    if (ne == 0) return 0;
    if (!elcon || !UH || !UHe) return -1;
    const size_t n = (size_t)ncu * ndf * ne;
    gather_uh_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(ncu, ndf, ne, elcon, UH, UHe);
    return launched();
}

int hdgx_globalassembly(const hdgx_bsr *A, const hdgx_assembly_map *map, int ncu, int npf, int nfe, const int *elcon,
                        const double *AE, const double *FE, double *Hg, double *Rg, hdgx_stream_t stream) {
    if (!A || !map || !elcon || !AE || !FE || !Hg || !Rg) return -1;
    if (A->bs != ncu * npf) return -2;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned g = (unsigned)(A->nnzb < (long long)sm_count() * 64 ? A->nnzb : (long long)sm_count() * 64);
    if (g < 1) g = 1;
    assemble_h_kernel<<<g, 256, 0, st>>>(ncu, npf, nfe, A->nnzb, map->blk_e, map->blk_ab, map->blk_row, A->colind,
                                         elcon, AE, Hg);
    const size_t n = (size_t)A->bs * A->nf;
    assemble_r_kernel<<<grid_for(n, 256), 256, 0, st>>>(ncu, npf, nfe, A->nf, map->face_e, map->face_a, elcon, FE, Rg);
    return launched();
}

int hdgx_matvec(const hdgx_bsr *A, const double *Hg, const double *x, double *y, hdgx_stream_t stream) {
    if (!A || !Hg || !x || !y) return -1;
    return trace_matvec(A, Hg, x, y, (cudaStream_t)stream);
}

int hdgx_bilu0_factor(const hdgx_bsr *A, double *Mg, int *status, hdgx_stream_t stream) {
    if (!A || !Mg || A->bs > 128 || A->bs < 1) return -1;
    cudaStream_t st = (cudaStream_t)stream;
    constexpr int NT = 256;
    const size_t smem = bilu_smem(A->bs);
    if (smem > 200 * 1024) return -3;
    if (A->ncolors == 0) {
        if (!A->sched) return -1;
        if (allow_dynamic_smem((const void *)bilu0_sched_factor_kernel<NT>, smem) != cudaSuccess)
            return -10;
        const int grid = resident_grid((const void *)bilu0_sched_factor_kernel<NT>, NT, smem, A->nf);
        sched_begin_kernel<<<1, 1, 0, st>>>(A->sched);
        bilu0_sched_factor_kernel<NT><<<grid, NT, smem, st>>>(A->bs, A->nf, A->color_rows, A->rowpts, A->colind, A->pos,
                                                              Mg, A->sched, status);
        return launched();
    }
    if (allow_dynamic_smem((const void *)bilu0_color_kernel<NT>, smem) != cudaSuccess)
        return -10;
    for (int c = 0; c < A->ncolors; c++) {
        const int r0 = A->color_ptr[c], nr = A->color_ptr[c + 1] - r0;
        if (nr <= 0) continue;
        unsigned grid = (unsigned)(nr < sm_count() * 8 ? nr : sm_count() * 8);
        bilu0_color_kernel<NT><<<grid, NT, smem, st>>>(A->bs, A->color_rows + r0, nr, A->rowpts, A->colind, A->pos, Mg,
                                                       status);
    }
    return launched();
}

int hdgx_bilu0_apply(const hdgx_bsr *A, const double *Mg, const double *x, double *v, double *work, hdgx_stream_t stream) {
    if (!A || !Mg || !x || !v || !work) return -1;
    return trace_bilu0_apply(A, Mg, x, work, v, (cudaStream_t)stream);
}

int hdgx_backsub(int npv, int nc, int ncu, int ndf, int ne, const int *elcon, const double *DUDG,
                 const double *DUDG_DUH, const double *DUH, double *DUDGT, hdgx_stream_t stream) {
    if (ne < 0 || !elcon || !DUDG || !DUDG_DUH || !DUH || !DUDGT) return -1;
    if (ne == 0) return 0;
    const int nh = ncu * ndf;
    unsigned g = (unsigned)(ne < sm_count() * 16 ? ne : sm_count() * 16);
    backsub_kernel<<<g, 128, sizeof(double) * nh, (cudaStream_t)stream>>>(ne, npv * nc, ncu, ndf, elcon, DUDG, DUDG_DUH,
                                                                          DUH, DUDGT);
    return launched();
}

int hdgx_block_norms(const hdgx_bsr *A, const double *Hg, double *C, hdgx_stream_t stream) {
    if (!A || !Hg || !C || A->bs > 128) return -1;
    const size_t need = sizeof(double) * (2 * (size_t)A->bs * A->bs + 130 + 8);
    if (need > 227 * 1024) return -3;
    if (allow_dynamic_smem((const void *)block_norms_kernel<256>, need) != cudaSuccess)
        return -10;
    const int grid = A->nf < sm_count() * 4 ? A->nf : sm_count() * 4;
    block_norms_kernel<256><<<grid, 256, need, (cudaStream_t)stream>>>(A->bs, A->nf, A->rowpts, Hg, C);
    return launched();
}

size_t hdgx_gmres_workspace_bytes(const hdgx_bsr *A, int restart) {
    if (!A || restart < 1) return 0;
    const size_t N = (size_t)A->bs * A->nf;
    const size_t m = (size_t)restart;
    return sizeof(double) * (N * (m + 1) + 3 * N + (m + 1) * m + 4 * (m + 1) + 8 + 2048 + 2 + m) + 256;
}

}  // extern "C"

namespace hdgx {

// GMRES steps launched between two host read-backs of the residual, for systems of at most
// kGmresBatchMaxN unknowns (larger ones read back after every step)
constexpr int kGmresBatch = 4;
constexpr size_t kGmresBatchMaxN = 262144;

int gmres_bilu0_run(const hdgx_bsr *A, const double *Hg, const double *Mg, const float *Mg32, const double *b,
                    double *x, int restart, double tol, int maxit, int *iters, int *flag, double *relres,
                    double *history, void *mem, cudaStream_t st) {
    auto prec = [&](const double *in, double *y, double *v) {
        return Mg32 ? trace_bilu0_apply_f32(A, Mg32, in, y, v, st) : trace_bilu0_apply(A, Mg, in, y, v, st);
    };
    const size_t N = (size_t)A->bs * A->nf;
    const int m = restart;
    double *V = (double *)mem;
    double *pb = V + N * (m + 1), *t = pb + N, *w2 = t + N;
    GmresState gs;
    gs.H = w2 + N;
    gs.cs = gs.H + (size_t)(m + 1) * m;
    gs.sn = gs.cs + (m + 1);
    gs.g = gs.sn + (m + 1);
    gs.y = gs.g + (m + 1);
    gs.scal = gs.y + (m + 1);
    double *part = gs.scal + 8;                   // [2048] partial sums
    unsigned *bar = reinterpret_cast<unsigned *>(part + 2048);   // grid barrier of the fused step
    int *bar_err = reinterpret_cast<int *>(bar + 1) + 1;         // [0] count, [1] generation, err
    gs.hist = part + 2048 + 2;                    // [m] residual norm after each step of a cycle
    cudaMemsetAsync(bar, 0, 3 * sizeof(unsigned), st);
    // host scalars on the stack (pageable copies are stream-ordered and, unlike freeing
    // pinned memory, never synchronise the other streams of the device)
    double h_scal[1 + kGmresBatch] = {};
    double *h_nrmb = h_scal, *h_hist = h_scal + 1;
    int rc = 0;
    const HostWaiter wait;                        // sleeps until the GPU is done in blocking mode
    // a failed launch or copy ends the solve at the next synchronisation: no further work is queued
    auto synced = [&]() {
        const cudaError_t e = cudaStreamSynchronize(st);
        if (e != cudaSuccess && !rc) rc = -1000 - (int)e;
        return rc == 0;
    };
    // pb = P^{-1} b, nrmb = |pb|
    if (int r = prec(b, t, pb)) rc = r;
    dot(N, pb, pb, gs.scal + 2, part, 1, st);
    wait(st);
    cudaMemcpyAsync(h_nrmb, gs.scal + 2, sizeof(double), cudaMemcpyDeviceToHost, st);
    synced();
    const double nrmb = *h_nrmb;
    int iter = 0, fl = 2;
    double res_rel = 0.0;
    if (!(nrmb > 0.0) || rc) { fl = rc ? 3 : 0; res_rel = 0.0; }
    while (fl == 2) {
        // r = pb - P^{-1} A x -> V[:,0] = r / beta
        if (int r = trace_matvec(A, Hg, x, t, st)) rc = rc ? rc : r;
        if (int r = prec(t, w2, V)) rc = rc ? rc : r;
        sub_kernel<<<grid_for(N, 256), 256, 0, st>>>(N, pb, V, V);
        dot(N, V, V, gs.scal + 0, part, 1, st);
        scale_div_kernel<<<grid_for(N, 256), 256, 0, st>>>(N, gs.scal + 0, V, V);
        gmres_init_kernel<<<1, 64, 0, st>>>(gs, m);
        int jdone = 0;
        bool stop = false;
        // Steps between host read-backs: each step's residual norm is recorded on the device and
        // read back `batch` steps at a time.  Steps past the one that stops write only what the
        // update does not read (H columns, g entries and V columns beyond jdone), so the result is
        // that of stopping there; one step at a time for large systems, whose steps are long.
        const int batch = N <= kGmresBatchMaxN ? kGmresBatch : 1;
        for (int j0 = 0; j0 < m && !stop;) {
            int kb = m - j0 < batch ? m - j0 : batch;
            if (kb > maxit - iter) kb = maxit - iter;
            for (int j = j0; j < j0 + kb; j++) {
                double *vj = V + N * j, *w = V + N * (j + 1);
                if (int r = trace_matvec(A, Hg, vj, t, st)) rc = rc ? rc : r;
                if (int r = prec(t, w2, w)) rc = rc ? rc : r;
                double *hc = gs.H + (size_t)(m + 1) * j;
                if (!mgs_fused(N, j + 1, V, w, hc, part, bar, bar_err, st)) {
                    for (int i = 0; i <= j; i++) {        // modified Gram-Schmidt (gmres_bilu0.m:59-63)
                        dot(N, V + N * i, w, hc + i, part, 0, st);
                        axpy_kernel<<<grid_for(N, 256), 256, 0, st>>>(N, hc + i, -1.0, V + N * i, w);
                    }
                    dot(N, w, w, hc + j + 1, part, 1, st);
                    scale_div_kernel<<<grid_for(N, 256), 256, 0, st>>>(N, hc + j + 1, w, w);
                }
                givens_kernel<<<1, 1, 0, st>>>(gs, m, j);
            }
            wait(st);
            cudaMemcpyAsync(h_hist, gs.hist + j0, sizeof(double) * kb, cudaMemcpyDeviceToHost, st);
            if (!synced()) { fl = 3; stop = true; break; }
            for (int k = 0; k < kb && !stop; k++) {
                res_rel = h_hist[k] / nrmb;
                if (history && iter < maxit) history[iter] = res_rel;
                iter++;
                jdone = j0 + k + 1;
                if (!isfinite(res_rel)) { fl = 3; stop = true; }
                else if (res_rel <= tol) { fl = 0; stop = true; }
                else if (iter >= maxit) { fl = 1; stop = true; }
            }
            j0 += kb;
        }
        if (rc) break;
        hess_solve_kernel<<<1, 1, 0, st>>>(gs, m, jdone);
        // x += V y  (y on the device; one axpy per basis vector)
        for (int i = 0; i < jdone; i++) axpy_kernel<<<grid_for(N, 256), 256, 0, st>>>(N, gs.y + i, 1.0, V + N * i, x);
        if (stop) break;
    }
    wait(st);
    synced();
    if (iters) *iters = iter;
    if (flag) *flag = fl;
    if (relres) *relres = res_rel;
    int mgs_err = 0;
    cudaMemcpyAsync(&mgs_err, bar_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    synced();
    int sched_err = 0;
    if (A->ncolors == 0 && A->sched) {
        cudaMemcpyAsync(&sched_err, A->sched + 2, sizeof(int), cudaMemcpyDeviceToHost, st);
        synced();
        if (sched_err) cudaMemsetAsync(A->sched + 2, 0, sizeof(int), st);
    }
    if (rc) return rc;
    if (cudaGetLastError() != cudaSuccess) return -12;
    if (sched_err) return -14;
    if (mgs_err) return -15;
    return 0;
}

}  // namespace hdgx

extern "C" {

int hdgx_gmres_bilu0(const hdgx_bsr *A, const double *Hg, const double *Mg, const double *b, double *x, int restart,
                     double tol, int maxit, int *iters, int *flag, double *relres, double *history, void *workspace,
                     hdgx_stream_t stream) {
    if (!A || !Hg || !Mg || !b || !x || restart < 1 || maxit < 1) return -1;
    cudaStream_t st = (cudaStream_t)stream;
    void *mem = workspace;
    bool own = false;
    if (!mem) {
        if (cudaMallocAsync(&mem, hdgx_gmres_workspace_bytes(A, restart), st) != cudaSuccess) return -13;
        own = true;
    }
    const int rc = gmres_bilu0_run(A, Hg, Mg, nullptr, b, x, restart, tol, maxit, iters, flag, relres, history, mem, st);
    if (own) cudaFreeAsync(mem, st);
    return rc;
}

int hdgx_bilu0_to_f32(const hdgx_bsr *A, const double *Mg, float *Mg32, hdgx_stream_t stream) {
    if (!A || !Mg || !Mg32 || A->bs < 1 || A->nnzb < 0) return -1;
    const size_t n = (size_t)A->bs * A->bs * (size_t)A->nnzb;
    if (n == 0) return 0;
    to_f32_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, Mg, Mg32);
    return launched();
}

int hdgx_gmres_bilu0_mixed(const hdgx_bsr *A, const double *Hg, const float *Mg32, const double *b, double *x,
                           int restart, double tol, int maxit, int *iters, int *flag, double *relres, double *history,
                           void *workspace, hdgx_stream_t stream) {
    if (!A || !Hg || !Mg32 || !b || !x || restart < 1 || maxit < 1) return -1;
    if (!A->sweep_plan || A->ncolors < 1) return -2;   // FP32 factors: level-scheduled sweeps only
    cudaStream_t st = (cudaStream_t)stream;
    void *mem = workspace;
    bool own = false;
    if (!mem) {
        if (cudaMallocAsync(&mem, hdgx_gmres_workspace_bytes(A, restart), st) != cudaSuccess) return -13;
        own = true;
    }
    const int rc = gmres_bilu0_run(A, Hg, nullptr, Mg32, b, x, restart, tol, maxit, iters, flag, relres, history, mem,
                                   st);
    if (own) cudaFreeAsync(mem, st);
    return rc;
}

}  // extern "C"

// computeMDFordering.m:21-161 with a lazy min-heap instead of the reference's linear min over
// all rows (same choices: smallest weight, ties to the lowest row).
extern "C" int hdgx_mdf_ordering(int nf, const long long *rowpts, const int *colind, const double *C, int *o2u,
                                 int *u2o) {
    if (nf < 0 || !rowpts || !colind || !C || !o2u || !u2o) return -1;
    std::vector<char> numbered(nf, 0);
    std::vector<double> w(nf, 0.0);
    auto pos_in_row = [&](int row, int col1) -> long long {
        for (long long k = rowpts[row]; k < rowpts[row + 1]; k++) if (colind[k] == col1) return k;
        return -1;
    };
    auto weight = [&](int k) {
        double acc = 0.0;
        for (long long ni = rowpts[k] + 1; ni < rowpts[k + 1]; ni++) {
            const int ri = colind[ni] - 1;
            if (numbered[ri]) continue;
            const long long ik = pos_in_row(ri, k + 1);
            if (ik < 0) continue;
            for (long long nj = rowpts[k] + 1; nj < rowpts[k + 1]; nj++) {
                if (nj == ni) continue;
                const int rj = colind[nj] - 1;
                if (numbered[rj]) continue;
                if (pos_in_row(ri, rj + 1) < 0) { const double d = C[ik] * C[nj]; acc += d * d; }
            }
        }
        return sqrt(acc);
    };
    typedef std::pair<double, int> E;
    std::priority_queue<E, std::vector<E>, std::greater<E>> heap;
    for (int k = 0; k < nf; k++) { w[k] = weight(k); heap.push(E(w[k], k)); }
    for (int l = 0; l < nf; l++) {
        int p = -1;
        while (!heap.empty()) {
            const E e = heap.top();
            heap.pop();
            if (!numbered[e.second] && e.first == w[e.second]) { p = e.second; break; }
        }
        if (p < 0) return -2;
        o2u[l] = p;
        numbered[p] = 1;
        for (long long e = rowpts[p] + 1; e < rowpts[p + 1]; e++) {
            const int k = colind[e] - 1;
            if (!numbered[k]) { w[k] = weight(k); heap.push(E(w[k], k)); }
        }
    }
    for (int i = 0; i < nf; i++) u2o[o2u[i]] = i;
    return 0;
}
