// capi.cu -- extern "C" entry points of libhdgx.so (declared in include/hdgx.h).
#include <cuda_runtime.h>
#include <math.h>
#include <mutex>
#include "hdgx_common.cuh"

namespace hdgx {
int elemental_launch(const hdgx_master *m, const hdgx_app *app, int ne, const double *dgnodes,
                     const int *bf, const double *UDG, const double *UH, const double *SH, double *AE,
                     double *FE, double *DUDG, double *DUDG_DUH, int *status, cudaStream_t st, bool mixed,
                     int grid);
int schur_launch(int qform, int nd, int npv, int ncu, int nc, int ndf, int ne, const double *M,
                 const double *C, const double *E, const double *BD, const double *F, const double *GK,
                 const double *H, const double *Rq, const double *Ru, const double *Rh, double *DUDG,
                 double *DUDG_DUH, double *AE, double *FE, int *status, cudaStream_t st);

__global__ void count_nonzero_kernel(const int *s, int n, int *out) {
    int c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) c += (s[i] != 0);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}
}  // namespace hdgx

extern "C" {

int hdgx_version(void) { return 10000; }

const char *hdgx_status_str(int code) {
    switch (code) {
        case 0: return "ok";
        case -1: return "invalid argument (null pointer or negative size)";
        case -2: return "inconsistent dimensions (nd, ncu, nc, npv, npf, nfe)";
        case -3: return "unsupported element size (shared-memory plan does not fit)";
        case -4: return "too many boundary indices";
        case -5: return "system too large for the allocation-free scratch (hdgx_gmres_bilu0_noalloc: 16 MiB)";
        case -10: return "cudaFuncSetAttribute failed";
        case -11: return "kernel does not fit on an SM";
        case -12: return "kernel launch failed";
        case -13: return "CUDA error while counting status";
        case -14: return "a flag-synchronised BILU(0) sweep gave up waiting (bounded spin)";
        case -15: return "the fused Gram-Schmidt step gave up waiting at a grid barrier (bounded spin)";
        default:
            if (code <= -1000) return cudaGetErrorString((cudaError_t)(-1000 - code));
            return "unknown status";
    }
}

int hdgx_status_count(const int *status, int n, hdgx_stream_t stream) {
    if (!status || n < 0) return -1;
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    int *d = nullptr, h = 0;
    if (cudaMallocAsync(&d, sizeof(int), st) != cudaSuccess) return -13;
    cudaMemsetAsync(d, 0, sizeof(int), st);
    int grid = (n + 255) / 256;
    if (grid > 1024) grid = 1024;
    hdgx::count_nonzero_kernel<<<grid, 256, 0, st>>>(status, n, d);
    cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return -13;
    return h;
}

}  // extern "C"

namespace {
// 0 when the elemental arguments are consistent (ne == 0 included), else the status code
int check_elemental(const hdgx_master *master, const hdgx_app *app, int ne, const double *dgnodes, const int *bf,
                    const double *UDG, const double *UH, const double *SH, const double *AE, const double *FE,
                    const double *DUDG, const double *DUDG_DUH) {
    if (!master || !app || ne < 0) return -1;
    if (ne == 0) return 0;
    if (!dgnodes || !bf || !UDG || !UH || !SH || !AE || !FE || !DUDG || !DUDG_DUH) return -1;
    if (!master->shapvt || !master->shapvg || !master->shapmv || !master->shapft || !master->shapfg ||
        !master->shapmf || !master->perm)
        return -1;
    const int nd = master->nd;
    if (app->nd != nd || app->ncu != nd + 2 || app->nc != (nd + 2) * (nd + 1) || master->nfe != nd + 1)
        return -2;
    if (app->localsolve != 1 || app->getdqdg != 1) return -2;
    if (app->nbnd < 0 || app->nbnd > HDGX_MAX_BND) return -4;
    return 0;
}

// Side streams of the bucketed launch, per device, created on the first call.
constexpr int kMaxFork = 8, kMaxDev = 64;
struct ForkSet {
    bool init = false;
    cudaStream_t s[kMaxFork];
    cudaEvent_t fork, join[kMaxFork];
};
std::mutex g_fork_mu;
ForkSet g_fork[kMaxDev];

int fork_set(ForkSet **out) {       // caller holds g_fork_mu
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return -12;
    ForkSet &f = g_fork[dev];
    if (!f.init) {
        if (cudaEventCreateWithFlags(&f.fork, cudaEventDisableTiming) != cudaSuccess) return -12;
        for (int k = 0; k < kMaxFork; k++) {
            if (cudaStreamCreateWithFlags(&f.s[k], cudaStreamNonBlocking) != cudaSuccess) return -12;
            if (cudaEventCreateWithFlags(&f.join[k], cudaEventDisableTiming) != cudaSuccess) return -12;
        }
        f.init = true;
    }
    *out = &f;
    return 0;
}
}  // namespace

extern "C" {

int hdgx_elemental(const hdgx_master *master, const hdgx_app *app, int ne, const double *dgnodes,
                   const int *bf, const double *UDG, const double *UH, const double *SH, double *AE,
                   double *FE, double *DUDG, double *DUDG_DUH, int *status, hdgx_stream_t stream) {
    if (int rc = check_elemental(master, app, ne, dgnodes, bf, UDG, UH, SH, AE, FE, DUDG, DUDG_DUH)) return rc;
    if (ne == 0) return 0;
    return hdgx::elemental_launch(master, app, ne, dgnodes, bf, UDG, UH, SH, AE, FE, DUDG, DUDG_DUH,
                                  status, (cudaStream_t)stream, false, 0);
}

int hdgx_elemental_mixed(const hdgx_master *master, const hdgx_app *app, int ne, const double *dgnodes,
                         const int *bf, const double *UDG, const double *UH, const double *SH, double *AE,
                         double *FE, double *DUDG, double *DUDG_DUH, int *status, hdgx_stream_t stream) {
    if (int rc = check_elemental(master, app, ne, dgnodes, bf, UDG, UH, SH, AE, FE, DUDG, DUDG_DUH)) return rc;
    if (ne == 0) return 0;
    return hdgx::elemental_launch(master, app, ne, dgnodes, bf, UDG, UH, SH, AE, FE, DUDG, DUDG_DUH,
                                  status, (cudaStream_t)stream, true, 0);
}

int hdgx_elemental_buckets(int nb, const hdgx_elem_bucket *b, int mixed, hdgx_stream_t stream) {
    if (nb < 0 || (nb > 0 && !b)) return -1;
    for (int k = 0; k < nb; k++) {
        const hdgx_elem_bucket &q = b[k];
        if (q.grid < 0) return -1;
        if (int rc = check_elemental(q.master, q.app, q.ne, q.dgnodes, q.bf, q.UDG, q.UH, q.SH, q.AE, q.FE, q.DUDG,
                                     q.DUDG_DUH))
            return rc;
    }
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> lk(g_fork_mu);
    ForkSet *fs = nullptr;
    if (int rc = fork_set(&fs)) return rc;
    if (cudaEventRecord(fs->fork, st) != cudaSuccess) return -12;
    bool used[kMaxFork] = {};
    int rc = 0;
    for (int k = 0; k < nb; k++) {
        const hdgx_elem_bucket &q = b[k];
        if (q.ne == 0) continue;
        const int si = k % kMaxFork;
        if (!used[si]) {
            if (cudaStreamWaitEvent(fs->s[si], fs->fork, 0) != cudaSuccess) rc = -12;
            used[si] = true;
        }
        const int r = hdgx::elemental_launch(q.master, q.app, q.ne, q.dgnodes, q.bf, q.UDG, q.UH, q.SH, q.AE, q.FE,
                                             q.DUDG, q.DUDG_DUH, q.status, fs->s[si], mixed != 0, q.grid);
        if (r && !rc) rc = r;
    }
    // join every side stream back into the caller's stream (also on failure, so that a
    // captured stream is never left forked)
    for (int si = 0; si < kMaxFork; si++) {
        if (!used[si]) continue;
        if (cudaEventRecord(fs->join[si], fs->s[si]) != cudaSuccess && !rc) rc = -12;
        if (cudaStreamWaitEvent(st, fs->join[si], 0) != cudaSuccess && !rc) rc = -12;
    }
    return rc;
}

int hdgx_schur_uq(int nd, int npv, int ncu, int ndf, int ne, const double *M, const double *C,
                  const double *E, const double *BD, const double *F, const double *GK, const double *H,
                  const double *Rq, const double *Ru, const double *Rh, double *DUDG, double *DUDG_DUH,
                  double *AE, double *FE, int *status, hdgx_stream_t stream) {
    if (ne < 0 || nd < 1 || npv < 1 || ncu < 1 || ndf < 1) return -1;
    if (ne == 0) return 0;
    if (!M || !C || !E || !BD || !F || !GK || !H || !Rq || !Ru || !Rh || !DUDG || !DUDG_DUH || !AE || !FE)
        return -1;
    return hdgx::schur_launch(1, nd, npv, ncu, ncu * (nd + 1), ndf, ne, M, C, E, BD, F, GK, H, Rq, Ru,
                              Rh, DUDG, DUDG_DUH, AE, FE, status, (cudaStream_t)stream);
}

int hdgx_schur_u(int npv, int ncu, int nc, int ndf, int ne, const double *BD, const double *F,
                 const double *GK, const double *H, const double *Ru, const double *Rh, double *DUDG,
                 double *DUDG_DUH, double *AE, double *FE, int *status, hdgx_stream_t stream) {
    if (ne < 0 || npv < 1 || ncu < 1 || nc < ncu || ndf < 1) return -1;
    if (ne == 0) return 0;
    if (!BD || !F || !GK || !H || !Ru || !Rh || !DUDG || !DUDG_DUH || !AE || !FE) return -1;
    return hdgx::schur_launch(0, 1, npv, ncu, nc, ndf, ne, nullptr, nullptr, nullptr, BD, F, GK, H,
                              nullptr, Ru, Rh, DUDG, DUDG_DUH, AE, FE, status, (cudaStream_t)stream);
}

}  // extern "C"
