// noalloc.cu -- GMRES on the condensed system without any device or pinned allocation.
//
// Some callers cannot call cudaMalloc / cudaMallocAsync / cudaMallocHost at solve time: a
// MEX or plugin host that owns the CUDA context and forbids allocations from the library
// (its allocator tracks every byte), a serving loop that must not touch the allocator on
// its latency path (an allocation can synchronise the device or fragment a pool), or code
// that has already reserved all device memory for its own arenas.  hdgx_gmres_bilu0 takes
// its Krylov basis from the stream-ordered allocator (or from a caller buffer);
// hdgx_gmres_bilu0_noalloc runs the very same solver (one shared implementation, the same
// matvec and BILU(0) sweep kernels, so the results are bitwise those of hdgx_gmres_bilu0)
// with every scratch array carved from one file-scope __device__ array of
// HDGX_NOALLOC_SCRATCH_BYTES (16 MiB) and host scalars on the stack.
//
// Limits and sharing:
//  * the scratch holds the basis V[N, restart+1] plus a few vectors, so it accepts systems
//    with hdgx_gmres_workspace_bytes(A, restart) <= 16 MiB (about N <= 88,000 unknowns at
//    restart 20); larger systems are rejected with status -5 before any work is queued;
//  * every GPU that loads the library holds the 16 MiB until the process exits.  With CUDA's
//    lazy module loading (the default) the module, and with it the array, is loaded on a
//    device at the first call there: that first call is the set-up, so make it (a warm-up
//    solve) before any latency-critical region and before any stream capture;
//  * every call shares the one array and it keeps the contents of the last call: calls
//    that overlap on the GPU (two streams, or two host threads on one device) race and
//    must be serialised by the caller.
#include <cuda_runtime.h>
#include <math.h>
#include <mutex>
#include "hdgx_common.cuh"
#include "trace_internal.cuh"

#define HDGX_NOALLOC_SCRATCH_BYTES (16u << 20)

// The allocation-free scratch.  In host code `g_noalloc_scratch` names a host-side stand-in,
// not device memory: only the address returned by cudaGetSymbolAddress may be handed to a
// kernel.  Device code in this file could name the array directly.
static __device__ __align__(256) unsigned char g_noalloc_scratch[HDGX_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct Resolved {
    unsigned long long ctx = 0;   // id of the context the address was resolved in (0: unknown)
    void *ptr = nullptr;
};
Resolved g_resolved[kMaxDevices];

// cuCtxGetId of the current context through the runtime's driver entry point (no link to the
// driver library); 0 when it is unavailable.
unsigned long long current_context_id() {
    typedef int (*GetCurrent)(void **);
    typedef int (*GetId)(void *, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void *f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (GetCurrent)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (GetId)f;
    });
    if (!get_current || !get_id) return 0;
    void *ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// Device address of the scratch array on the current device.  It is resolved with
// cudaGetSymbolAddress once per device and context: a context recreated after
// cudaDeviceReset reloads the module at another address, so the cache is keyed on the
// context id (and resolved on every call where that id cannot be read).
int scratch_address(void **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -13;
    const unsigned long long ctx = current_context_id();
    std::lock_guard<std::mutex> lk(g_mu);
    Resolved &r = g_resolved[dev];
    if (!r.ptr || ctx == 0 || r.ctx != ctx) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return -13;
        r.ptr = p;
        r.ctx = ctx;
    }
    *out = r.ptr;
    return 0;
}

}  // namespace

extern "C" int hdgx_gmres_bilu0_noalloc(const hdgx_bsr *A, const double *Hg, const double *Mg, const double *b,
                                        double *x, int restart, double tol, int maxit, int *iters, int *flag,
                                        double *relres, double *history, hdgx_stream_t stream) {
    if (!A || !Hg || !Mg || !b || !x || restart < 1 || maxit < 1) return -1;
    if (A->ncolors == 0 && !A->sched) return -1;     // flag-scheduled sweeps need the caller's sched array
    const size_t need = hdgx_gmres_workspace_bytes(A, restart);
    if (need == 0 || need > HDGX_NOALLOC_SCRATCH_BYTES) return -5;
    void *base = nullptr;
    if (int rc = scratch_address(&base)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // The array keeps the previous call's contents: clear it up to the end of this call's
    // workspace, so that nothing of an earlier solve (Hessenberg columns, rotations, the grid
    // barrier of the fused Gram-Schmidt step) can leak into this one.
    if (cudaMemsetAsync(base, 0, need, st) != cudaSuccess) return -12;
    return hdgx::gmres_bilu0_run(A, Hg, Mg, nullptr, b, x, restart, tol, maxit, iters, flag, relres, history, base,
                                 st);
}
