// capi.cu -- extern "C" entry points of libhdgx.so (declared in include/hdgx.h).
#include <cuda_runtime.h>
#include <math.h>
#include "hdgx_common.cuh"

namespace hdgx {
int elemental_launch(const hdgx_master *m, const hdgx_app *app, int ne, const double *dgnodes,
                     const int *bf, const double *UDG, const double *UH, const double *SH, double *AE,
                     double *FE, double *DUDG, double *DUDG_DUH, int *status, cudaStream_t st, bool mixed);
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

int hdgx_elemental(const hdgx_master *master, const hdgx_app *app, int ne, const double *dgnodes,
                   const int *bf, const double *UDG, const double *UH, const double *SH, double *AE,
                   double *FE, double *DUDG, double *DUDG_DUH, int *status, hdgx_stream_t stream) {
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
    return hdgx::elemental_launch(master, app, ne, dgnodes, bf, UDG, UH, SH, AE, FE, DUDG, DUDG_DUH,
                                  status, (cudaStream_t)stream, false);
}

int hdgx_elemental_mixed(const hdgx_master *master, const hdgx_app *app, int ne, const double *dgnodes,
                         const int *bf, const double *UDG, const double *UH, const double *SH, double *AE,
                         double *FE, double *DUDG, double *DUDG_DUH, int *status, hdgx_stream_t stream) {
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
    return hdgx::elemental_launch(master, app, ne, dgnodes, bf, UDG, UH, SH, AE, FE, DUDG, DUDG_DUH,
                                  status, (cudaStream_t)stream, true);
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
