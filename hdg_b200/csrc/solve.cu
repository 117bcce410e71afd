// solve.cu -- hdgx_solve: the Newton loop of kernel/hdg_solve.m:84-176 in native code.
//
// One call takes the master element, the app, a mesh whose per-element arrays are already on
// the device and the state (UDG, UH on the device), and runs Newton to the requested relative
// residual: assembly (hdg_assemble.m: trace gather, elemental kernel, block-CSR gather),
// BILU(0)-GMRES on the condensed system (in the minimum-discarded-fill order of
// computeMDFordering.m by default), back-substitution (hdg_solve.m:119-121) and the halving line
// search of hdg_solve.m:144-163.  The host-side set-up it needs (element -> block assembly map,
// elimination order, level schedule, sweep records) is built here from the mesh's host
// connectivity.  Every device buffer comes from the stream-ordered allocator and is released
// before returning, into a private pool that keeps up to 8 GiB of freed memory for the next
// solve.
#include <cuda_runtime.h>
#include <math.h>
#include <algorithm>
#include <mutex>
#include <vector>
#include "hdgx_common.cuh"

namespace hdgx {

int elemental_check_master(const hdgx_master *m);
int combiner_attach(hdgx_combiner *c, uint64_t key);
void combiner_detach(hdgx_combiner *c, uint64_t key);
int combiner_key(hdgx_combiner *c, const hdgx_master *m, const hdgx_app *app, cudaStream_t st, uint64_t *key);
int combiner_submit(hdgx_combiner *c, const hdgx_elem_bucket &b, uint64_t key, cudaStream_t st);

// y = x0 + alpha * d   (the line-search update hdg_solve.m:146-147)
__global__ void add_scaled_kernel(size_t n, const double *__restrict__ x0, double alpha, const double *__restrict__ d,
                                  double *__restrict__ y) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        y[t] = x0[t] + alpha * d[t];
}

__global__ void dot_partial_kernel(size_t, const double *, const double *, double *);
__global__ void dot_final_kernel(int, const double *, double *, int);

namespace {

struct HostPlan {
    // assembly map
    std::vector<int> blk_e, blk_ab, blk_row, face_e, face_a;
    // elimination order
    int ncolors = 0;
    std::vector<int> color_ptr, color_rows, pos;
    std::vector<int> sweep;
    int sweep_maxd = 0;
};

long long find_block(const long long *rowpts, const int *colind, int row, int col0) {
    for (long long k = rowpts[row]; k < rowpts[row + 1]; k++)
        if (colind[k] - 1 == col0) return k;
    return -1;
}

// globalassembly.m:24-37 visits blocks element by element; record the (element, local face
// pair) contributions of every block and the (element, local face) pairs of every face.
int build_assembly_map(int ne, int nfe, int nf, const int *t2f, const long long *rowpts, const int *colind,
                       HostPlan &hp) {
    const long long nnzb = rowpts[nf];
    hp.blk_e.assign(2 * nnzb, -1);
    hp.blk_ab.assign(2 * nnzb, 0);
    hp.blk_row.resize(nnzb);
    hp.face_e.assign(2 * (size_t)nf, -1);
    hp.face_a.assign(2 * (size_t)nf, 0);
    std::vector<int> fill(nnzb, 0), ffill(nf, 0);
    for (int i = 0; i < nf; i++)
        for (long long k = rowpts[i]; k < rowpts[i + 1]; k++) hp.blk_row[k] = i;
    for (int e = 0; e < ne; e++)
        for (int a = 0; a < nfe; a++) {
            const int i = abs(t2f[e + (size_t)ne * a]) - 1;
            if (i < 0 || i >= nf || ffill[i] >= 2) return -2;
            hp.face_e[2 * i + ffill[i]] = e;
            hp.face_a[2 * i + ffill[i]] = a;
            ffill[i]++;
            for (int b = 0; b < nfe; b++) {
                const long long k = find_block(rowpts, colind, i, abs(t2f[e + (size_t)ne * b]) - 1);
                if (k < 0 || fill[k] >= 2) return -2;
                hp.blk_e[2 * k + fill[k]] = e;
                hp.blk_ab[2 * k + fill[k]] = a | (b << 8);
                fill[k]++;
            }
        }
    return 0;
}

// greedy colouring in natural row order (rows of one colour share no block)
void build_multicolor(int nf, const long long *rowpts, const int *colind, HostPlan &hp) {
    std::vector<int> color(nf, -1);
    int ncol = 0;
    std::vector<char> used;
    for (int i = 0; i < nf; i++) {
        used.assign(ncol + 2, 0);
        for (long long k = rowpts[i] + 1; k < rowpts[i + 1]; k++) {
            const int c = color[colind[k] - 1];
            if (c >= 0) used[c] = 1;
        }
        int c = 0;
        while (used[c]) c++;
        color[i] = c;
        ncol = std::max(ncol, c + 1);
    }
    hp.ncolors = ncol;
    hp.color_ptr.assign(ncol + 1, 0);
    for (int i = 0; i < nf; i++) hp.color_ptr[color[i] + 1]++;
    for (int c = 0; c < ncol; c++) hp.color_ptr[c + 1] += hp.color_ptr[c];
    std::vector<int> next(hp.color_ptr.begin(), hp.color_ptr.end() - 1);
    hp.color_rows.resize(nf);
    hp.pos.resize(nf);
    for (int i = 0; i < nf; i++) hp.color_rows[next[color[i]]++] = i;
    for (int q = 0; q < nf; q++) hp.pos[hp.color_rows[q]] = q;
    hp.sweep.clear();
    hp.sweep_maxd = 0;
}

// A sequential order o2u eliminated level by level: level(i) = 1 + max level of the
// neighbours eliminated before i; rows of a level share no block, and ILU(0) factors depend
// only on which of two coupled rows comes first, so the factors are the sequential order's.
// Level schedule of the sequential elimination order o2u: level(i) = 1 + the largest level of
// the neighbours eliminated before i; rows grouped by level, by position inside a level.
// level_ptr [nlev + 1] (room for nf + 1), rows [nf]; returns nlev.
int level_schedule(int nf, const long long *rowpts, const int *colind, const int *o2u, const int *u2o,
                   int *level_ptr, int *rows) {
    std::vector<int> lev(nf, 0);
    int nlev = 0;
    for (int j = 0; j < nf; j++) {
        const int i = o2u[j];
        int L = -1;
        for (long long k = rowpts[i] + 1; k < rowpts[i + 1]; k++) {
            const int c = colind[k] - 1;
            if (u2o[c] < j) L = std::max(L, lev[c]);
        }
        lev[i] = L + 1;
        nlev = std::max(nlev, L + 2);
    }
    for (int c = 0; c <= nlev; c++) level_ptr[c] = 0;
    for (int i = 0; i < nf; i++) level_ptr[lev[i] + 1]++;
    for (int c = 0; c < nlev; c++) level_ptr[c + 1] += level_ptr[c];
    std::vector<int> next(level_ptr, level_ptr + nlev);
    for (int j = 0; j < nf; j++) {                  // by level, then by position
        const int i = o2u[j];
        rows[next[lev[i]]++] = i;
    }
    return nlev;
}

// Record width of the one-launch sweeps: 4 or 6 (block, column) pairs per side, 0 when a row
// has more than 6 off-diagonal blocks (no single-launch plan).
int sweep_width(int nf, const long long *rowpts) {
    int dmax = 0;
    for (int i = 0; i < nf; i++) dmax = std::max<int>(dmax, (int)(rowpts[i + 1] - rowpts[i] - 1));
    return dmax > 6 ? 0 : (dmax <= 4 ? 4 : 6);
}

// The single-launch sweep plan: [nlev + 1] level offsets, then per slot q of rows the record
// (row i, its diagonal block rowpts[i], maxd (block, column) pairs of the neighbours eliminated
// before i, maxd pairs of those eliminated after i), -1 padded, 0-based, neighbours in CSR order.
void sweep_records(int nf, const long long *rowpts, const int *colind, int nlev, const int *level_ptr,
                   const int *rows, const int *pos, int maxd, int *plan) {
    const int RW = 2 + 4 * maxd;
    for (int c = 0; c <= nlev; c++) plan[c] = level_ptr[c];
    for (size_t t = 0; t < (size_t)nf * RW; t++) plan[nlev + 1 + t] = -1;
    for (int q = 0; q < nf; q++) {
        int *R = plan + (nlev + 1) + (size_t)q * RW;
        const int i = rows[q];
        R[0] = i;
        R[1] = (int)rowpts[i];
        int nb = 0, na = 0;
        for (long long k = rowpts[i] + 1; k < rowpts[i + 1]; k++) {
            const int j = colind[k] - 1;
            if (pos[j] < pos[i]) { R[2 + 2 * nb] = (int)k; R[3 + 2 * nb] = j; nb++; }
            else { R[2 + 2 * maxd + 2 * na] = (int)k; R[3 + 2 * maxd + 2 * na] = j; na++; }
        }
    }
}

void build_levels(int nf, const long long *rowpts, const int *colind, const std::vector<int> &o2u,
                  const std::vector<int> &u2o, HostPlan &hp) {
    std::vector<int> ptr(nf + 1);
    hp.color_rows.resize(nf);
    const int nlev = level_schedule(nf, rowpts, colind, o2u.data(), u2o.data(), ptr.data(), hp.color_rows.data());
    hp.ncolors = nlev;
    hp.color_ptr.assign(ptr.begin(), ptr.begin() + nlev + 1);
    hp.pos = u2o;
    // fixed-width dependency records of the one-launch sweeps (hdgx_bsr.sweep_plan)
    const int maxd = sweep_width(nf, rowpts);
    hp.sweep_maxd = maxd;
    if (!maxd) { hp.sweep.clear(); return; }
    hp.sweep.resize((size_t)(nlev + 1) + (size_t)nf * (2 + 4 * maxd));
    sweep_records(nf, rowpts, colind, nlev, hp.color_ptr.data(), hp.color_rows.data(), hp.pos.data(), maxd,
                  hp.sweep.data());
}

// A private stream-ordered memory pool per device.  Freed blocks stay in the pool up to
// kKeepBytes across synchronisations (the default pool returns everything to the driver at
// every synchronisation, and remapping it on the next solve costs more than a small solve).
constexpr int kMaxDev = 64;
constexpr unsigned long long kKeepBytes = 8ull << 30;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxDev] = {};

cudaMemPool_t solve_pool() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) return nullptr;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pool[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
        unsigned long long keep = kKeepBytes;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        g_pool[dev] = p;
    }
    return g_pool[dev];
}

// device buffers from the stream-ordered allocator, released together
struct DevPool {
    cudaStream_t st;
    cudaMemPool_t pool;
    std::vector<void *> ptrs;
    bool failed = false;
    explicit DevPool(cudaStream_t s) : st(s), pool(solve_pool()) { if (!pool) failed = true; }
    template <class T>
    T *get(size_t n) {
        void *p = nullptr;
        if (n == 0) n = 1;
        if (!pool || cudaMallocFromPoolAsync(&p, sizeof(T) * n, pool, st) != cudaSuccess) { failed = true; return nullptr; }
        ptrs.push_back(p);
        return (T *)p;
    }
    template <class T>
    T *upload(const std::vector<T> &v) {
        T *p = get<T>(v.size());
        if (p && !v.empty()) cudaMemcpyAsync(p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, st);
        return p;
    }
    ~DevPool() {
        for (void *p : ptrs) cudaFreeAsync(p, st);
    }
};

// |x| into out[0] (two kernels, no synchronisation)
void norm2_launch(size_t n, const double *x, double *part, double *out, cudaStream_t st) {
    const int nsm = sm_count_of(current_device());
    size_t g = (n + 255) / 256;
    if (g > (size_t)nsm * 8) g = (size_t)nsm * 8;
    if (g > 1024) g = 1024;
    if (g < 1) g = 1;
    dot_partial_kernel<<<(unsigned)g, 256, 0, st>>>(n, x, x, part);
    dot_final_kernel<<<1, 256, 0, st>>>((int)g, part, out, 1);
}

double read_scalar(const double *d, cudaStream_t st, const HostWaiter &wait) {
    double h = 0.0;
    wait(st);
    cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    return h;
}

// The assembly chain of one Newton solve as a CUDA graph, launched for every assembly after the
// first: the inputs and outputs sit at fixed device addresses for the whole solve.
struct ChainGraph {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~ChainGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (g) cudaGraphDestroy(g);
    }
};

}  // namespace

// the same private pool for the other entry points that stage data on the device
cudaMemPool_t device_pool() { return solve_pool(); }
}  // namespace hdgx

using namespace hdgx;

namespace {

// A solve's membership of a combiner.
struct CombinerLink {
    hdgx_combiner *c = nullptr;
    uint64_t key = 0;
    ~CombinerLink() {
        if (c) combiner_detach(c, key);
    }
};

int solve_impl(const hdgx_master *m, const hdgx_app *app, const hdgx_mesh *mesh, double *UDG, double *UH,
               const double *SH, const hdgx_solve_opts *opts, hdgx_solve_report *rep, hdgx_combiner *comb,
               hdgx_stream_t stream) {
    if (!m || !app || !mesh || !UDG || !UH || !SH || !opts) return -1;
    if (!mesh->dgnodes || !mesh->bf || !mesh->elcon || !mesh->t2f || !mesh->rowpts || !mesh->colind) return -1;
    const int ne = mesh->ne, nf = mesh->nf;
    if (ne < 1 || nf < 1 || opts->restart < 1 || opts->maxiter < 0 || opts->gmres_maxit < 1) return -1;
    if (app->getdqdg != 1) return -2;    // the native loop keeps q in the local solve (getdqdg = 1)
    if (int rc = hdgx::elemental_check_master(m)) return rc;   // before any set-up or allocation
    if (opts->ordering != 0 && opts->ordering != 1) return -1;
    if (comb && opts->mixed) return -2;                         // shared launches are FP64
    cudaStream_t st = (cudaStream_t)stream;
    CombinerLink link;
    if (comb) {
        if (int rc = combiner_key(comb, m, app, st, &link.key)) return rc;
        if (int rc = combiner_attach(comb, link.key)) return rc;
        link.c = comb;
    }
    const int npv = m->npv, npf = m->npf, nfe = m->nfe, ncu = app->ncu, nc = app->nc;
    const int ndf = npf * nfe, bs = ncu * npf;
    const long long nnzb = mesh->rowpts[nf];
    const size_t nU = (size_t)npv * nc * ne, nH = (size_t)bs * nf;

    HostPlan hp;
    if (int rc = build_assembly_map(ne, nfe, nf, mesh->t2f, mesh->rowpts, mesh->colind, hp)) return rc;
    if (opts->ordering == 1) build_multicolor(nf, mesh->rowpts, mesh->colind, hp);

    DevPool pool(st);
    long long *d_rowpts = pool.upload(std::vector<long long>(mesh->rowpts, mesh->rowpts + nf + 1));
    int *d_colind = pool.upload(std::vector<int>(mesh->colind, mesh->colind + nnzb));
    hdgx_assembly_map map;
    map.blk_e = pool.upload(hp.blk_e);
    map.blk_ab = pool.upload(hp.blk_ab);
    map.blk_row = pool.upload(hp.blk_row);
    map.face_e = pool.upload(hp.face_e);
    map.face_a = pool.upload(hp.face_a);
    double *UHe = pool.get<double>((size_t)ncu * ndf * ne);
    double *AE = pool.get<double>((size_t)ncu * ndf * ncu * ndf * ne), *FE = pool.get<double>((size_t)ncu * ndf * ne);
    double *DUDG = pool.get<double>(nU), *DUDG_DUH = pool.get<double>(nU * ncu * ndf);
    double *Hg = pool.get<double>((size_t)bs * bs * nnzb), *Mg = pool.get<double>((size_t)bs * bs * nnzb);
    double *Rg = pool.get<double>(nH), *DUH = pool.get<double>(nH), *DUDGT = pool.get<double>(nU);
    double *UDG0 = pool.get<double>(nU), *UH0 = pool.get<double>(nH);
    double *part = pool.get<double>(1024 + 8);
    int *status = pool.get<int>(ne);
    // hdg_solve.m:62-63: without the wave formulation the q part of SH is zero
    double *SHz = pool.get<double>(nU);
    if (pool.failed) return -13;
    cudaMemcpyAsync(SHz, SH, sizeof(double) * nU, cudaMemcpyDeviceToDevice, st);
    cudaMemset2DAsync(SHz + (size_t)npv * ncu, sizeof(double) * npv * nc, 0, sizeof(double) * npv * (nc - ncu), ne, st);
    SH = SHz;

    hdgx_bsr A = {};
    A.nf = nf;
    A.bs = bs;
    A.nnzb = nnzb;
    A.rowpts = d_rowpts;
    A.colind = d_colind;
    auto set_order = [&]() {
        A.ncolors = hp.ncolors;
        A.color_ptr = hp.color_ptr.data();
        A.color_rows = pool.upload(hp.color_rows);
        A.pos = pool.upload(hp.pos);
        A.sched = nullptr;
        A.sweep_plan = hp.sweep.empty() ? nullptr : pool.upload(hp.sweep);
        A.sweep_maxd = hp.sweep_maxd;
    };
    if (opts->ordering == 1) set_order();
    void *ws = pool.get<unsigned char>(hdgx_gmres_workspace_bytes(&A, opts->restart));
    if (pool.failed) return -13;
    const int nsm = [] { int d = 0, n = 0; cudaGetDevice(&d); cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d); return n > 0 ? n : 1; }();
    const unsigned gU = (unsigned)std::min<size_t>((nU + 255) / 256, (size_t)nsm * 8);
    const unsigned gH = (unsigned)std::min<size_t>((nH + 255) / 256, (size_t)nsm * 8);

    // hdg_assemble.m (trace gather, elemental kernel, block-CSR gather) and |F| into part[1024]
    auto assemble_chain = [&]() -> int {
        int rc = hdgx_gather_uh(ncu, ndf, ne, mesh->elcon, UH, UHe, stream);
        if (rc) return rc;
        if (comb) {
            const hdgx_elem_bucket b = {m, app, ne, mesh->dgnodes, mesh->bf, UDG, UHe, SH, AE, FE, DUDG, DUDG_DUH,
                                        status, 0};
            rc = combiner_submit(comb, b, link.key, st);
        } else {
            rc = opts->mixed ? hdgx_elemental_mixed(m, app, ne, mesh->dgnodes, mesh->bf, UDG, UHe, SH, AE, FE, DUDG,
                                                    DUDG_DUH, status, stream)
                             : hdgx_elemental(m, app, ne, mesh->dgnodes, mesh->bf, UDG, UHe, SH, AE, FE, DUDG,
                                              DUDG_DUH, status, stream);
        }
        if (rc) return rc;
        rc = hdgx_globalassembly(&A, &map, ncu, npf, nfe, mesh->elcon, AE, FE, Hg, Rg, stream);
        if (rc) return rc;
        norm2_launch(nH, Rg, part, part + 1024, st);
        return 0;
    };
    // After the first assembly (which also does every kernel's first-use set-up), the chain is
    // captured once into a graph on the solve's stream (thread-local capture; only on a
    // non-blocking stream, which the legacy default stream never waits on, and not with a
    // combiner, whose batching synchronises on the host).  A capture that fails leaves the
    // plain launches in use.
    const HostWaiter wait;                        // how the host waits for the read-backs
    ChainGraph chain;
    bool chain_tried = comb != nullptr;
    int graph_runs = 0;
    auto capture_chain = [&]() {
        chain_tried = true;
        unsigned flags = 0;
        if (!st || cudaStreamGetFlags(st, &flags) != cudaSuccess || !(flags & cudaStreamNonBlocking)) return;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        const int rc = assemble_chain();
        const cudaError_t e = cudaStreamEndCapture(st, &chain.g);
        if (rc || e != cudaSuccess || !chain.g || cudaGraphInstantiate(&chain.exec, chain.g, 0) != cudaSuccess) {
            if (chain.g) cudaGraphDestroy(chain.g);
            chain.g = nullptr;
            chain.exec = nullptr;
            cudaGetLastError();
        }
    };
    // returns |F| or a negative status
    auto assemble = [&](double *res) -> int {
        if (chain.exec) {
            if (cudaGraphLaunch(chain.exec, st) != cudaSuccess) return -12;
            graph_runs++;
        } else if (int rc = assemble_chain()) {
            return rc;
        }
        *res = read_scalar(part + 1024, st, wait);
        if (!chain_tried) capture_chain();
        return 0;
    };

    hdgx_solve_report r = {};
    double F = 0.0;
    if (int rc = assemble(&F)) return rc;
    const double F0 = F;
    r.residuals[0] = F;
    double rel = 1.0;
    int it = 0;
    bool ordered = opts->ordering == 1;
    float *Mg32 = nullptr;                           // FP32 factors (mixed precision), allocated once
    while (rel > opts->tol && it < opts->maxiter && it < HDGX_SOLVE_MAXIT) {
        if (!ordered) {
            // computeMDFordering.m on the first assembled matrix
            double *C = pool.get<double>(nnzb);
            if (!C) return -13;
            if (int rc = hdgx_block_norms(&A, Hg, C, stream)) return rc;
            std::vector<double> Ch(nnzb);
            wait(st);
            cudaMemcpyAsync(Ch.data(), C, sizeof(double) * nnzb, cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
            std::vector<int> o2u(nf), u2o(nf);
            if (int rc = hdgx_mdf_ordering(nf, mesh->rowpts, mesh->colind, Ch.data(), o2u.data(), u2o.data())) return rc;
            build_levels(nf, mesh->rowpts, mesh->colind, o2u, u2o, hp);
            set_order();
            if (pool.failed) return -13;
            ordered = true;
        }
        cudaMemcpyAsync(Mg, Hg, sizeof(double) * bs * bs * nnzb, cudaMemcpyDeviceToDevice, st);
        if (int rc = hdgx_bilu0_factor(&A, Mg, nullptr, stream)) return rc;
        cudaMemsetAsync(DUH, 0, sizeof(double) * nH, st);
        int gi = 0, gfl = 0;
        double grr = 0.0;
        // mixed precision: the preconditioner's factors in FP32 where the level sweeps run them
        const bool f32 = opts->mixed && A.sweep_plan && A.ncolors > 0;
        if (f32 && !Mg32 && !(Mg32 = pool.get<float>((size_t)bs * bs * nnzb))) return -13;
        if (f32 && (hdgx_bilu0_to_f32(&A, Mg, Mg32, stream) != 0)) return -12;
        if (int rc = f32 ? hdgx_gmres_bilu0_mixed(&A, Hg, Mg32, Rg, DUH, opts->restart, opts->gmres_tol,
                                                  opts->gmres_maxit, &gi, &gfl, &grr, nullptr, ws, stream)
                         : hdgx_gmres_bilu0(&A, Hg, Mg, Rg, DUH, opts->restart, opts->gmres_tol, opts->gmres_maxit,
                                            &gi, &gfl, &grr, nullptr, ws, stream))
            return rc;
        r.gmres_iters[it] = gi;
        r.gmres_relres[it] = grr;
        if (int rc = hdgx_backsub(npv, nc, ncu, ndf, ne, mesh->elcon, DUDG, DUDG_DUH, DUH, DUDGT, stream)) return rc;
        cudaMemcpyAsync(UDG0, UDG, sizeof(double) * nU, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(UH0, UH, sizeof(double) * nH, cudaMemcpyDeviceToDevice, st);
        const double duh0 = F;
        double alfa = 1.0;
        for (;;) {                                   // hdg_solve.m:144-163
            add_scaled_kernel<<<gU, 256, 0, st>>>(nU, UDG0, alfa, DUDGT, UDG);
            add_scaled_kernel<<<gH, 256, 0, st>>>(nH, UH0, alfa, DUH, UH);
            if (int rc = assemble(&F)) return rc;
            if (F > duh0) {
                alfa /= 2;
                if (alfa < 1e-2) break;
            } else {
                break;
            }
        }
        r.alphas[it] = alfa;
        it++;
        r.residuals[it] = F;
        rel = F0 > 0.0 ? F / F0 : 0.0;
    }
    wait(st);
    cudaStreamSynchronize(st);
    r.iterations = it;
    r.converged = rel <= opts->tol;
    r.ncolors = A.ncolors;
    r.graph_assemblies = graph_runs;
    if (rep) *rep = r;
    return cudaGetLastError() == cudaSuccess ? 0 : -12;
}

}  // namespace

extern "C" int hdgx_solve(const hdgx_master *m, const hdgx_app *app, const hdgx_mesh *mesh, double *UDG, double *UH,
                          const double *SH, const hdgx_solve_opts *opts, hdgx_solve_report *rep,
                          hdgx_stream_t stream) {
    return solve_impl(m, app, mesh, UDG, UH, SH, opts, rep, nullptr, stream);
}

extern "C" int hdgx_solve_combined(const hdgx_master *m, const hdgx_app *app, const hdgx_mesh *mesh, double *UDG,
                                   double *UH, const double *SH, const hdgx_solve_opts *opts, hdgx_solve_report *rep,
                                   hdgx_combiner *combiner, hdgx_stream_t stream) {
    if (!combiner) return -1;
    return solve_impl(m, app, mesh, UDG, UH, SH, opts, rep, combiner, stream);
}

extern "C" int hdgx_level_schedule(int nf, const long long *rowpts, const int *colind, const int *o2u, const int *u2o,
                                   int *level_ptr, int *rows) {
    if (nf < 0 || !rowpts || !colind || !o2u || !u2o || !level_ptr || !rows) return -1;
    for (int j = 0; j < nf; j++)
        if (o2u[j] < 0 || o2u[j] >= nf || u2o[o2u[j]] != j) return -1;   // not a permutation pair
    return hdgx::level_schedule(nf, rowpts, colind, o2u, u2o, level_ptr, rows);
}

extern "C" int hdgx_sweep_plan(int nf, const long long *rowpts, const int *colind, int nlev, const int *level_ptr,
                               const int *rows, const int *pos, int *plan, int *maxd) {
    if (nf < 0 || nlev < 0 || !rowpts || !colind || !level_ptr || !rows || !pos || !maxd) return -1;
    *maxd = hdgx::sweep_width(nf, rowpts);
    if (*maxd == 0 || !plan) return 0;             // no plan, or the width asked for alone
    hdgx::sweep_records(nf, rowpts, colind, nlev, level_ptr, rows, pos, *maxd, plan);
    return 0;
}
