// noalloc.cu -- GMRES on the condensed system without any device or pinned allocation.
//
// Some callers cannot call cudaMalloc / cudaMallocAsync / cudaMallocHost at solve time: a
// MEX or plugin host that owns the CUDA context and forbids allocations from the library
// (its allocator tracks every byte), a serving loop that must not touch the allocator on
// its latency path (an allocation can synchronise the device or fragment a pool), or code
// that has already reserved all device memory for its own arenas.  hdgx_gmres_bilu0 takes
// its Krylov basis from the stream-ordered allocator (or from a caller buffer) and pins two
// host scalars; hdgx_gmres_bilu0_noalloc runs the same algorithm with every scratch array
// carved from one file-scope __device__ array of HDGX_NOALLOC_SCRATCH_BYTES (16 MiB) and
// host scalars on the stack.
//
// Limits and sharing:
//  * the scratch holds the basis V[N, restart+1] plus a few vectors, so it accepts systems
//    with hdgx_gmres_workspace_bytes(A, restart) <= 16 MiB (about N <= 88,000 unknowns at
//    restart 20); larger systems are rejected with status -5 before any work is queued;
//  * every GPU that loads the library holds the 16 MiB until the process exits;
//  * every call shares the one array and it keeps the contents of the last call: calls
//    that overlap on the GPU (two streams, or two host threads on one device) race and
//    must be serialised by the caller;
//  * the first call on each device resolves the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it; make that first call
//    before any stream capture.
#include <cuda_runtime.h>
#include <math.h>
#include <mutex>
#include "hdgx_common.cuh"

#define HDGX_NOALLOC_SCRATCH_BYTES (16u << 20)

// The allocation-free scratch.  In host code `g_noalloc_scratch` names a host-side stand-in,
// not device memory: only the address returned by cudaGetSymbolAddress may be handed to a
// kernel.  Device code in this file could name the array directly.
static __device__ __align__(256) unsigned char g_noalloc_scratch[HDGX_NOALLOC_SCRATCH_BYTES];

namespace hdgx {
__global__ void bsr_matvec_kernel(int, int, const long long *, const int *, const double *, const double *, double *);
__global__ void bilu0_fwd_kernel(int, const int *, int, const long long *, const int *, const int *, const double *,
                                 const double *, double *);
__global__ void bilu0_bwd_kernel(int, const int *, int, const long long *, const int *, const int *, const double *,
                                 const double *, double *);
__global__ void dot_partial_kernel(size_t, const double *, const double *, double *);
__global__ void dot_final_kernel(int, const double *, double *, int);
__global__ void axpy_kernel(size_t, const double *, double, const double *, double *);
__global__ void scale_div_kernel(size_t, const double *, const double *, double *);
__global__ void sub_kernel(size_t, const double *, const double *, double *);
struct GmresState {
    double *H, *cs, *sn, *g, *y;
    double *scal;
};
__global__ void givens_kernel(GmresState, int, int);
__global__ void hess_solve_kernel(GmresState, int, int);
__global__ void gmres_init_kernel(GmresState, int);
}  // namespace hdgx

using namespace hdgx;

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_dev_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (set-up once per device).
int scratch_address(void **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -13;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_dev_ptr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return -13;
        g_dev_ptr[dev] = p;
    }
    *out = g_dev_ptr[dev];
    return 0;
}

int n_sm() {
    int d = 0, n = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d);
    return n > 0 ? n : 1;
}

unsigned grid_n(size_t n, int threads, int nsm) {
    size_t g = (n + threads - 1) / threads, cap = (size_t)nsm * 8;
    if (g > cap) g = cap;
    return (unsigned)(g < 1 ? 1 : g);
}

void mv(const hdgx_bsr *A, const double *Hg, const double *x, double *y, cudaStream_t st, int nsm) {
    bsr_matvec_kernel<<<grid_n((size_t)A->nf * 32, 256, nsm), 256, 0, st>>>(A->nf, A->bs, A->rowpts, A->colind, Hg, x, y);
}

void prec(const hdgx_bsr *A, const double *Mg, const double *x, double *y, double *v, cudaStream_t st) {
    const int threads = 256, warps = threads / 32;
    for (int c = 0; c < A->ncolors; c++) {
        const int r0 = A->color_ptr[c], nr = A->color_ptr[c + 1] - r0;
        if (nr > 0)
            bilu0_fwd_kernel<<<(nr + warps - 1) / warps, threads, 0, st>>>(A->bs, A->color_rows + r0, nr, A->rowpts,
                                                                          A->colind, A->pos, Mg, x, y);
    }
    for (int c = A->ncolors - 1; c >= 0; c--) {
        const int r0 = A->color_ptr[c], nr = A->color_ptr[c + 1] - r0;
        if (nr > 0)
            bilu0_bwd_kernel<<<(nr + warps - 1) / warps, threads, sizeof(double) * warps * A->bs, st>>>(
                A->bs, A->color_rows + r0, nr, A->rowpts, A->colind, A->pos, Mg, y, v);
    }
}

void dotp(size_t n, const double *a, const double *b, double *out, double *part, int do_sqrt, cudaStream_t st, int nsm) {
    unsigned g = grid_n(n, 256, nsm);
    if (g > 1024) g = 1024;
    dot_partial_kernel<<<g, 256, 0, st>>>(n, a, b, part);
    dot_final_kernel<<<1, 256, 0, st>>>((int)g, part, out, do_sqrt);
}

}  // namespace

extern "C" int hdgx_gmres_bilu0_noalloc(const hdgx_bsr *A, const double *Hg, const double *Mg, const double *b,
                                        double *x, int restart, double tol, int maxit, int *iters, int *flag,
                                        double *relres, double *history, hdgx_stream_t stream) {
    if (!A || !Hg || !Mg || !b || !x || restart < 1 || maxit < 1) return -1;
    if (A->ncolors < 1) return -1;   // the flag-scheduled (sequential-order) sweeps are not offered here
    const size_t need = hdgx_gmres_workspace_bytes(A, restart);
    if (need == 0 || need > HDGX_NOALLOC_SCRATCH_BYTES) return -5;
    void *base = nullptr;
    if (int rc = scratch_address(&base)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int nsm = n_sm();
    const size_t N = (size_t)A->bs * A->nf;
    const int m = restart;
    double *V = (double *)base;
    double *pb = V + N * (m + 1), *t = pb + N, *w2 = t + N;
    GmresState gs;
    gs.H = w2 + N;
    gs.cs = gs.H + (size_t)(m + 1) * m;
    gs.sn = gs.cs + (m + 1);
    gs.g = gs.sn + (m + 1);
    gs.y = gs.g + (m + 1);
    gs.scal = gs.y + (m + 1);
    double *part = gs.scal + 8;
    // The array keeps the previous call's contents: clear the Hessenberg / rotation / scalar
    // state so nothing of an earlier solve can leak into this one.
    cudaMemsetAsync(gs.H, 0, sizeof(double) * ((size_t)(m + 1) * m + 4 * (m + 1) + 8), st);
    double h_nrmb = 0.0, h_res = 0.0;
    prec(A, Mg, b, t, pb, st);
    dotp(N, pb, pb, gs.scal + 2, part, 1, st, nsm);
    cudaMemcpyAsync(&h_nrmb, gs.scal + 2, sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    const double nrmb = h_nrmb;
    int iter = 0, fl = 2;
    double res_rel = 0.0;
    if (!(nrmb > 0.0)) fl = 0;
    while (fl == 2) {
        mv(A, Hg, x, t, st, nsm);
        prec(A, Mg, t, w2, V, st);
        sub_kernel<<<grid_n(N, 256, nsm), 256, 0, st>>>(N, pb, V, V);
        dotp(N, V, V, gs.scal + 0, part, 1, st, nsm);
        scale_div_kernel<<<grid_n(N, 256, nsm), 256, 0, st>>>(N, gs.scal + 0, V, V);
        gmres_init_kernel<<<1, 64, 0, st>>>(gs, m);
        int jdone = 0;
        bool stop = false;
        for (int j = 0; j < m; j++) {
            double *vj = V + N * j, *w = V + N * (j + 1);
            mv(A, Hg, vj, t, st, nsm);
            prec(A, Mg, t, w2, w, st);
            double *hc = gs.H + (size_t)(m + 1) * j;
            for (int i = 0; i <= j; i++) {
                dotp(N, V + N * i, w, hc + i, part, 0, st, nsm);
                axpy_kernel<<<grid_n(N, 256, nsm), 256, 0, st>>>(N, hc + i, -1.0, V + N * i, w);
            }
            dotp(N, w, w, hc + j + 1, part, 1, st, nsm);
            scale_div_kernel<<<grid_n(N, 256, nsm), 256, 0, st>>>(N, hc + j + 1, w, w);
            givens_kernel<<<1, 1, 0, st>>>(gs, m, j);
            cudaMemcpyAsync(&h_res, gs.scal + 1, sizeof(double), cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
            res_rel = h_res / nrmb;
            if (history && iter < maxit) history[iter] = res_rel;
            iter++;
            jdone = j + 1;
            if (!isfinite(res_rel)) { fl = 3; stop = true; break; }
            if (res_rel <= tol) { fl = 0; stop = true; break; }
            if (iter >= maxit) { fl = 1; stop = true; break; }
        }
        hess_solve_kernel<<<1, 1, 0, st>>>(gs, m, jdone);
        for (int i = 0; i < jdone; i++) axpy_kernel<<<grid_n(N, 256, nsm), 256, 0, st>>>(N, gs.y + i, 1.0, V + N * i, x);
        if (stop) break;
    }
    cudaStreamSynchronize(st);
    if (iters) *iters = iter;
    if (flag) *flag = fl;
    if (relres) *relres = res_rel;
    return cudaGetLastError() == cudaSuccess ? 0 : -12;
}
