// capi.cu -- extern "C" entry points of libhdgx.so (declared in include/hdgx.h).
#include <cuda_runtime.h>
#include <math.h>
#include <atomic>
#include <mutex>
#include <utility>
#include <vector>
#include "hdgx_common.cuh"

namespace hdgx {
int elemental_launch(const hdgx_master *m, const hdgx_app *app, int ne, const double *dgnodes,
                     const int *bf, const double *UDG, const double *UH, const double *SH, double *AE,
                     double *FE, double *DUDG, double *DUDG_DUH, int *status, cudaStream_t st, bool mixed,
                     int grid, double *QDG = nullptr, double *RU = nullptr);
cudaMemPool_t device_pool();
int elemental_check_master(const hdgx_master *m);
int elemental_launch_shared(int nb, const hdgx_elem_bucket *b, cudaStream_t st, int grid);
int elemental_shared_max_segments();
int schur_adjoint_launch(int qform, int nd, int npv, int ncu, int nc, int ndf, int ne, const double *M,
                         const double *C, const double *E, const double *BD, const double *F, const double *GK,
                         const double *H, const double *Rq, const double *Ru, const double *Rh, double *DUDG,
                         double *DUDG_DUH, double *AE, double *FE, int *status, cudaStream_t st);
int schur_launch(int qform, int nd, int npv, int ncu, int nc, int ndf, int ne, const double *M,
                 const double *C, const double *E, const double *BD, const double *F, const double *GK,
                 const double *H, const double *Rq, const double *Ru, const double *Rh, double *DUDG,
                 double *DUDG_DUH, double *AE, double *FE, int *status, cudaStream_t st);

std::atomic<int> g_host_wait{0};

// Blocking-synchronisation events, per device, created on demand and reused
static std::mutex g_wait_mu;
static std::vector<std::pair<int, cudaEvent_t>> g_wait_free;

cudaEvent_t host_wait_acquire() {
    if (g_host_wait.load(std::memory_order_relaxed) != 1) return nullptr;
    const int dev = current_device();
    {
        std::lock_guard<std::mutex> lk(g_wait_mu);
        for (size_t i = 0; i < g_wait_free.size(); i++)
            if (g_wait_free[i].first == dev) {
                cudaEvent_t e = g_wait_free[i].second;
                g_wait_free[i] = g_wait_free.back();
                g_wait_free.pop_back();
                return e;
            }
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreateWithFlags(&e, cudaEventBlockingSync | cudaEventDisableTiming) != cudaSuccess) return nullptr;
    return e;
}

void host_wait_release(cudaEvent_t ev) {
    if (!ev) return;
    std::lock_guard<std::mutex> lk(g_wait_mu);
    g_wait_free.emplace_back(current_device(), ev);
}

__global__ void count_nonzero_kernel(const int *s, int n, int *out) {
    int c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) c += (s[i] != 0);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}
}  // namespace hdgx

extern "C" {

int hdgx_version(void) { return 10000; }

int hdgx_set_host_wait(int mode) {
    if (mode != 0 && mode != 1) return -1;
    hdgx::g_host_wait.store(mode);
    return 0;
}

int hdgx_get_host_wait(void) { return hdgx::g_host_wait.load(); }

const char *hdgx_status_str(int code) {
    switch (code) {
        case 0: return "ok";
        case -1: return "invalid argument (null pointer or negative size)";
        case -2: return "inconsistent dimensions (nd, ncu, nc, npv, npf, nfe)";
        case -3: return "unsupported element: (nd, porder) not compiled, or master tables (npv, npf, ngv, ngf) "
                        "other than those of quadrature order pgauss = 2 porder";
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
    if (app->localsolve != 1 || (app->getdqdg != 0 && app->getdqdg != 1)) return -2;
    if (app->nbnd < 0 || app->nbnd > HDGX_MAX_BND) return -4;
    return hdgx::elemental_check_master(master);     // -3: tables of another (porder, pgauss)
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

int hdgx_getq(const hdgx_master *master, const hdgx_app *app, int ne, const double *dgnodes, const int *bf,
              const double *UDG, const double *UH, const double *SH, double *QDG, int *status,
              hdgx_stream_t stream) {
    if (!master || !app || ne < 0) return -1;
    if (ne == 0) return 0;
    if (!dgnodes || !bf || !UDG || !UH || !QDG) return -1;
    if (!master->shapvt || !master->shapvg || !master->shapmv || !master->shapft || !master->shapfg ||
        !master->shapmf || !master->perm)
        return -1;
    const int nd = master->nd;
    if (app->nd != nd || app->ncu != nd + 2 || app->nc != (nd + 2) * (nd + 1) || master->nfe != nd + 1) return -2;
    if (!(app->fc_q != 0.0)) return -1;
    return hdgx::elemental_launch(master, app, ne, dgnodes, bf, UDG, UH, SH, nullptr, nullptr, nullptr, nullptr,
                                  status, (cudaStream_t)stream, false, 0, QDG);
}

int hdgx_residual(const hdgx_master *master, const hdgx_app *app, int ne, const double *dgnodes, const int *bf,
                  const double *UDG, const double *UH, const double *SH, double *Ru, int *status,
                  hdgx_stream_t stream) {
    if (!master || !app || ne < 0) return -1;
    if (ne == 0) return 0;
    if (!dgnodes || !bf || !UDG || !UH || !Ru) return -1;
    if (!master->shapvt || !master->shapvg || !master->shapmv || !master->shapft || !master->shapfg ||
        !master->shapmf || !master->perm)
        return -1;
    const int nd = master->nd;
    if (app->nd != nd || app->ncu != nd + 2 || app->nc != (nd + 2) * (nd + 1) || master->nfe != nd + 1) return -2;
    if (app->nbnd < 0 || app->nbnd > HDGX_MAX_BND) return -4;
    if (!(app->fc_q != 0.0)) return -1;
    return hdgx::elemental_launch(master, app, ne, dgnodes, bf, UDG, UH, SH, nullptr, nullptr, nullptr, nullptr,
                                  status, (cudaStream_t)stream, false, 0, nullptr, Ru);
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

int hdgx_elemental_shared(int nb, const hdgx_elem_bucket *b, int grid, hdgx_stream_t stream) {
    if (nb < 0 || (nb > 0 && !b) || grid < 0) return -1;
    if (nb == 0) return 0;
    if (nb > hdgx::elemental_shared_max_segments()) return -5;
    for (int k = 0; k < nb; k++) {
        const hdgx_elem_bucket &q = b[k];
        if (int rc = check_elemental(q.master, q.app, q.ne, q.dgnodes, q.bf, q.UDG, q.UH, q.SH, q.AE, q.FE, q.DUDG,
                                     q.DUDG_DUH))
            return rc;
    }
    return hdgx::elemental_launch_shared(nb, b, (cudaStream_t)stream, grid);
}

int hdgx_elemental_shared_max(void) { return hdgx::elemental_shared_max_segments(); }

// Host-array form: the elements go through two device staging sets in chunks, and chunk c's
// upload (stream s_in), chunk c-1's kernel (the caller's stream) and chunk c-2's download
// (stream s_out) run at the same time.  Set b = c % 2 is reused by chunk c + 2 only after
// chunk c's kernel has read its inputs (upload waits on ev_k[b]) and chunk c's download has
// read its outputs (kernel waits on ev_out[b]).
int hdgx_elemental_host(const hdgx_master *master, const hdgx_app *app, int ne, const double *dgnodes,
                        const int *bf, const double *UDG, const double *UH, const double *SH, double *AE,
                        double *FE, double *DUDG, double *DUDG_DUH, int *status, int mixed, int chunk,
                        hdgx_stream_t stream) {
    if (int rc = check_elemental(master, app, ne, dgnodes, bf, UDG, UH, SH, AE, FE, DUDG, DUDG_DUH)) return rc;
    if (chunk < 0) return -1;
    if (ne == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t npv = master->npv, nd = master->nd, nfe = master->nfe, nc = app->nc, ncu = app->ncu;
    const size_t ndf = (size_t)master->npf * nfe;
    // doubles (ints for bf, status) per element of every array, in argument order
    const size_t nco = app->getdqdg ? nc : ncu;       // components of DUDG / DUDG_DUH
    const size_t n_x = npv * nd, n_u = npv * nc, n_h = ncu * ndf, n_ae = n_h * n_h, n_o = npv * nco,
                 n_dd = n_o * n_h;
    if (chunk == 0) chunk = ne < 16 * 1024 ? (ne < 1024 ? ne : 1024) : (ne + 15) / 16;
    if (chunk > ne) chunk = ne;
    // one staging set: every array of `chunk` elements, each on a 256-byte boundary
    const size_t dbl[8] = {n_x, n_u, n_h, n_u, n_ae, n_h, n_o, n_dd}, ints[2] = {nfe, 1};
    auto rnd = [](size_t bytes) { return (bytes + 255) & ~(size_t)255; };
    size_t set_bytes = 0;
    for (size_t d : dbl) set_bytes += rnd(sizeof(double) * d * chunk);
    for (size_t d : ints) set_bytes += rnd(sizeof(int) * d * chunk);
    cudaMemPool_t pool = hdgx::device_pool();
    if (!pool) return -12;
    unsigned char *stage = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync((void **)&stage, 2 * set_bytes, pool, st);
    if (e != cudaSuccess) return -1000 - (int)e;
    struct Set { double *x, *u, *h, *s, *ae, *fe, *dd, *ddh; int *bf, *status; } set[2];
    for (int b = 0; b < 2; b++) {
        unsigned char *p = stage + b * set_bytes;
        double **dp[8] = {&set[b].x, &set[b].u, &set[b].h, &set[b].s, &set[b].ae, &set[b].fe, &set[b].dd, &set[b].ddh};
        for (int k = 0; k < 8; k++) { *dp[k] = (double *)p; p += rnd(sizeof(double) * dbl[k] * chunk); }
        set[b].bf = (int *)p;
        p += rnd(sizeof(int) * nfe * chunk);
        set[b].status = (int *)p;
    }
    cudaStream_t s_in = nullptr, s_out = nullptr;
    cudaEvent_t ev_start = nullptr, ev_done = nullptr, ev_in[2] = {}, ev_k[2] = {}, ev_out[2] = {};
    int rc = 0;
    auto ok = [&](cudaError_t r) { if (r != cudaSuccess && !rc) rc = -1000 - (int)r; return rc == 0; };
    ok(cudaStreamCreateWithFlags(&s_in, cudaStreamNonBlocking));
    ok(cudaStreamCreateWithFlags(&s_out, cudaStreamNonBlocking));
    ok(cudaEventCreateWithFlags(&ev_start, cudaEventDisableTiming));
    ok(cudaEventCreateWithFlags(&ev_done, cudaEventDisableTiming));
    for (int b = 0; b < 2; b++) {
        ok(cudaEventCreateWithFlags(&ev_in[b], cudaEventDisableTiming));
        ok(cudaEventCreateWithFlags(&ev_k[b], cudaEventDisableTiming));
        ok(cudaEventCreateWithFlags(&ev_out[b], cudaEventDisableTiming));
    }
    if (rc == 0) {
        ok(cudaEventRecord(ev_start, st));                  // the staging allocation is ordered on st
        ok(cudaStreamWaitEvent(s_in, ev_start, 0));
        ok(cudaStreamWaitEvent(s_out, ev_start, 0));
        const int nch = (ne + chunk - 1) / chunk;
        for (int c = 0; c < nch && rc == 0; c++) {
            const int b = c & 1;
            const size_t e0 = (size_t)c * chunk;
            const int n = (int)((size_t)ne - e0 < (size_t)chunk ? (size_t)ne - e0 : (size_t)chunk);
            const Set &S = set[b];
            auto h2d = [&](void *dst, const void *src, size_t per) {
                return ok(cudaMemcpyAsync(dst, (const unsigned char *)src + per * e0, per * n, cudaMemcpyHostToDevice, s_in));
            };
            auto d2h = [&](void *dst, const void *src, size_t per) {
                return ok(cudaMemcpyAsync((unsigned char *)dst + per * e0, src, per * n, cudaMemcpyDeviceToHost, s_out));
            };
            if (c >= 2) ok(cudaStreamWaitEvent(s_in, ev_k[b], 0));
            h2d(S.x, dgnodes, sizeof(double) * n_x);
            h2d(S.bf, bf, sizeof(int) * nfe);
            h2d(S.u, UDG, sizeof(double) * n_u);
            h2d(S.h, UH, sizeof(double) * n_h);
            h2d(S.s, SH, sizeof(double) * n_u);
            ok(cudaEventRecord(ev_in[b], s_in));
            ok(cudaStreamWaitEvent(st, ev_in[b], 0));
            if (c >= 2) ok(cudaStreamWaitEvent(st, ev_out[b], 0));
            if (rc) break;
            const int r = hdgx::elemental_launch(master, app, n, S.x, S.bf, S.u, S.h, S.s, S.ae, S.fe, S.dd, S.ddh,
                                                 status ? S.status : nullptr, st, mixed != 0, 0);
            if (r) { rc = r; break; }
            ok(cudaEventRecord(ev_k[b], st));
            ok(cudaStreamWaitEvent(s_out, ev_k[b], 0));
            d2h(AE, S.ae, sizeof(double) * n_ae);
            d2h(FE, S.fe, sizeof(double) * n_h);
            d2h(DUDG, S.dd, sizeof(double) * n_o);
            d2h(DUDG_DUH, S.ddh, sizeof(double) * n_dd);
            if (status) d2h(status, S.status, sizeof(int));
            ok(cudaEventRecord(ev_out[b], s_out));
        }
        // join the copy streams back into st (also after a failure), then release the staging
        cudaEventRecord(ev_done, s_in);
        cudaStreamWaitEvent(st, ev_done, 0);
        cudaEventRecord(ev_done, s_out);
        cudaStreamWaitEvent(st, ev_done, 0);
    }
    cudaFreeAsync(stage, st);
    ok(cudaStreamSynchronize(st));
    if (s_in) cudaStreamDestroy(s_in);
    if (s_out) cudaStreamDestroy(s_out);
    for (cudaEvent_t ev : {ev_start, ev_done, ev_in[0], ev_in[1], ev_k[0], ev_k[1], ev_out[0], ev_out[1]})
        if (ev) cudaEventDestroy(ev);
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

int hdgx_schur_uq_adjoint(int nd, int npv, int ncu, int ndf, int ne, const double *M, const double *C,
                          const double *E, const double *BD, const double *F, const double *GK, const double *H,
                          const double *Rq, const double *Ru, const double *Rh, double *DUDG, double *DUDG_DUH,
                          double *AE, double *FE, int *status, hdgx_stream_t stream) {
    if (ne < 0 || nd < 1 || npv < 1 || ncu < 1 || ndf < 1) return -1;
    if (ne == 0) return 0;
    if (!M || !C || !E || !BD || !F || !GK || !H || !Rq || !Ru || !Rh || !DUDG || !DUDG_DUH || !AE || !FE)
        return -1;
    return hdgx::schur_adjoint_launch(1, nd, npv, ncu, ncu * (nd + 1), ndf, ne, M, C, E, BD, F, GK, H, Rq, Ru,
                                      Rh, DUDG, DUDG_DUH, AE, FE, status, (cudaStream_t)stream);
}

int hdgx_schur_u_adjoint(int npv, int ncu, int nc, int ndf, int ne, const double *BD, const double *F,
                         const double *GK, const double *H, const double *Ru, const double *Rh, double *DUDG,
                         double *DUDG_DUH, double *AE, double *FE, int *status, hdgx_stream_t stream) {
    if (ne < 0 || npv < 1 || ncu < 1 || nc < ncu || ndf < 1) return -1;
    if (ne == 0) return 0;
    if (!BD || !F || !GK || !H || !Ru || !Rh || !DUDG || !DUDG_DUH || !AE || !FE) return -1;
    return hdgx::schur_adjoint_launch(0, 1, npv, ncu, nc, ndf, ne, nullptr, nullptr, nullptr, BD, F, GK, H,
                                      nullptr, Ru, Rh, DUDG, DUDG_DUH, AE, FE, status, (cudaStream_t)stream);
}

}  // extern "C"
