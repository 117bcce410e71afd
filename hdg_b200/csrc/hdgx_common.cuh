// hdgx_common.cuh -- shared device helpers for the HDG elemental kernels (sm_100a, FP64).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/hdgx.h"
#include <atomic>
#include <map>
#include <mutex>
#include <utility>

namespace hdgx {
// Raise a kernel's dynamic shared-memory limit to at least `bytes` on the current device.
// The limit is a process-wide attribute of the function: host threads that launch the same
// kernel for different block sizes would otherwise lower it under one another's launches
// (which then fail with "invalid argument").  The limit only ever grows here, under a lock.
inline cudaError_t allow_dynamic_smem(const void *fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, size_t> granted;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    size_t &g = granted[std::make_pair(dev, fn)];
    if (bytes <= g) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) g = bytes;
    return e;
}

// Device attributes that every launch needs, cached per device ordinal (host threads of a
// server may launch concurrently and on different devices; the values never change for a
// device within a process).
constexpr int kMaxDevices = 64;
inline int current_device() {
    int dev = 0;
    return cudaGetDevice(&dev) == cudaSuccess ? dev : 0;
}
inline int sm_count_of(int dev) {
    static std::atomic<int> cache[kMaxDevices];
    if (dev < 0 || dev >= kMaxDevices) dev = 0;
    int n = cache[dev].load(std::memory_order_relaxed);
    if (n <= 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) return 1;
        cache[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

// How a host thread waits for the GPU where a solve reads a scalar back (GMRES residual, |F|):
// mode 0 (default) as CUDA does by default, the thread spinning in the copy or synchronisation;
// mode 1 (hdgx_set_host_wait) the thread first sleeps on a blocking-synchronisation event of a
// pooled set until the GPU has reached that point, so that many concurrent solves do not keep as
// many cores busy spinning.  Events come from a per-device pool (no create / destroy per solve).
cudaEvent_t host_wait_acquire();         // nullptr in mode 0
void host_wait_release(cudaEvent_t ev);
struct HostWaiter {
    cudaEvent_t ev;
    HostWaiter() : ev(host_wait_acquire()) {}
    ~HostWaiter() { host_wait_release(ev); }
    HostWaiter(const HostWaiter &) = delete;
    HostWaiter &operator=(const HostWaiter &) = delete;
    // returns once the work queued on st so far has completed (mode 1), at once otherwise
    void operator()(cudaStream_t st) const {
        if (ev && cudaEventRecord(ev, st) == cudaSuccess) cudaEventSynchronize(ev);
    }
};
}  // namespace hdgx

namespace hdgx {

// Physics constants derived from hdgx_app.param = [gam, epslm, Re, Pr, Minf, tau].
struct PhysConst {
    double gam1, rinv, kap, tau;
};

// ------------------------------------------------------------------ dual numbers
// value + one directional derivative; each thread differentiates along one seed.
struct D1 {
    double v, d;
};
__device__ __forceinline__ D1 dc(double v) { return {v, 0.0}; }
__device__ __forceinline__ D1 operator+(D1 a, D1 b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ D1 operator-(D1 a, D1 b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ D1 operator*(D1 a, D1 b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ D1 operator*(D1 a, double s) { return {a.v * s, a.d * s}; }
__device__ __forceinline__ D1 operator/(D1 a, D1 b) {
    double ib = 1.0 / b.v;
    double q = a.v * ib;
    return {q, (a.d - q * b.d) * ib};
}

// Compressible Navier-Stokes flux in all ND directions at one point (Euler when rinv = 0).
// u[NCU] conserved state, q[NCU*ND] gradient slots (component fastest, the reference's
// sign convention q = -grad u is carried through unchanged).  f[a + NCU*j].
// Physics: application/FM/ns/flux2d.m / flux3d.m (flux_ns2d.c / flux_ns3d.c).
template <int ND>
__device__ __forceinline__ void ns_flux(const PhysConst &pc, const D1 *u, const D1 *q, D1 *f) {
    constexpr int NCU = ND + 2;
    const D1 r = u[0], rE = u[NCU - 1];
    D1 vel[ND];
    D1 ke = dc(0.0);
#pragma unroll
    for (int i = 0; i < ND; i++) {
        vel[i] = u[1 + i] / r;
        ke = ke + vel[i] * u[1 + i];
    }
    const D1 p = (rE - ke * 0.5) * pc.gam1;
    const D1 h = (rE + p) / r;
    if (pc.rinv == 0.0) {
#pragma unroll
        for (int j = 0; j < ND; j++) {
            f[0 + NCU * j] = u[1 + j];
#pragma unroll
            for (int i = 0; i < ND; i++) {
                D1 t = u[1 + i] * vel[j];
                if (i == j) t = t + p;
                f[(1 + i) + NCU * j] = t;
            }
            f[(NCU - 1) + NCU * j] = h * u[1 + j];
        }
        return;
    }
    const D1 ri = dc(1.0) / r;
    D1 gv[ND][ND];
#pragma unroll
    for (int i = 0; i < ND; i++)
#pragma unroll
        for (int j = 0; j < ND; j++) gv[i][j] = (q[(1 + i) + NCU * j] - vel[i] * q[NCU * j]) * ri;
    D1 div = dc(0.0);
#pragma unroll
    for (int i = 0; i < ND; i++) div = div + gv[i][i];
    D1 v2 = dc(0.0);
#pragma unroll
    for (int i = 0; i < ND; i++) v2 = v2 + vel[i] * vel[i];
#pragma unroll
    for (int j = 0; j < ND; j++) {
        D1 tauj[ND];
#pragma unroll
        for (int i = 0; i < ND; i++) {
            D1 t = gv[i][j] + gv[j][i];
            if (i == j) t = t - div * (2.0 / 3.0);
            tauj[i] = t * pc.rinv;
        }
        D1 vdv = dc(0.0);
#pragma unroll
        for (int i = 0; i < ND; i++) vdv = vdv + vel[i] * gv[i][j];
        const D1 qr = q[NCU * j];
        const D1 pj = (q[(NCU - 1) + NCU * j] - v2 * 0.5 * qr - r * vdv) * pc.gam1;
        const D1 Tj = (pj * r - p * qr) / (r * r);
        f[0 + NCU * j] = u[1 + j];
        D1 e = h * u[1 + j];
#pragma unroll
        for (int i = 0; i < ND; i++) {
            D1 t = u[1 + i] * vel[j] + tauj[i];
            if (i == j) t = t + p;
            f[(1 + i) + NCU * j] = t;
            e = e + vel[i] * tauj[i];
        }
        f[(NCU - 1) + NCU * j] = e + Tj * pc.kap;
    }
}

// ------------------------------------------------------------ boundary fluxes (fbou)
__device__ __forceinline__ D1 dsqrt(D1 a) {
    const double r = sqrt(a.v);
    return {r, a.d * 0.5 / r};
}
__device__ __forceinline__ D1 dabs(D1 a) { return a.v < 0.0 ? D1{-a.v, -a.d} : a; }   // sign(0) = 1
__device__ __forceinline__ D1 dscale(D1 a, double s) { return {a.v * s, a.d * s}; }

// Constants of the boundary fluxes: family (0: application/FM/ns/fbou.m and fbou3d.m,
// 1: application/FM/euler/fbou.m), gam, the entropy-fix width eps = param[1], Minf^2.
struct FbouConst {
    int fam;
    double gam, eps, m2;
};

// y = A x for the Roe matrices of getan.m at the state m (absolute = false: the normal flux
// Jacobian A_n; true: |A_n|, with |l| replaced by (|l|^2/(eps c) + eps c)/2 where |l| < eps c).
// A = l3 I + r1 w1' + r2 w2' (r1 = [1, v, h], r2 = [0, n, un], w1 = (s1-l3) gam1/c^2 P + s2/c N,
// w2 = s2 gam1/c P + (s1-l3) N, P = [|v|^2/2, -v, 1], N = [-un, n, 0], l1,2,3 = un+c, un-c, un),
// applied through its two rank-one terms instead of being formed.
template <int ND>
__device__ __forceinline__ void roe_apply(double gam, double eps, const double *nl, const D1 *m, bool absolute,
                                          const D1 *x, D1 *y) {
    constexpr int NCU = ND + 2;
    const double gam1 = gam - 1.0;
    const D1 r = m[0];
    D1 v[ND], un = dc(0.0), af = dc(0.0);
#pragma unroll
    for (int i = 0; i < ND; i++) {
        v[i] = m[1 + i] / r;
        un = un + dscale(v[i], nl[i]);
        af = af + dscale(v[i] * v[i], 0.5);
    }
    const D1 p = dscale(m[NCU - 1] - r * af, gam1);
    const D1 c = dsqrt(dscale(p, gam) / r);
    const D1 h = (m[NCU - 1] + p) / r;
    D1 l[3] = {un + c, un - c, un};
    if (absolute) {
        const D1 ec = dscale(c, eps);
#pragma unroll
        for (int i = 0; i < 3; i++) {
            l[i] = dabs(l[i]);
            if (eps > 0.0 && l[i].v < ec.v) l[i] = dscale(l[i] * l[i] / ec + ec, 0.5);
        }
    }
    const D1 s1 = dscale(l[0] + l[1], 0.5), s2 = dscale(l[0] - l[1], 0.5), d = s1 - l[2];
    const D1 k1 = dscale(d, gam1) / (c * c), k2 = s2 / c, k3 = dscale(k2, gam1);
    D1 Px = af * x[0] + x[NCU - 1], Nx = dc(0.0) - un * x[0];
#pragma unroll
    for (int i = 0; i < ND; i++) {
        Px = Px - v[i] * x[1 + i];
        Nx = Nx + dscale(x[1 + i], nl[i]);
    }
    const D1 w1 = k1 * Px + k2 * Nx, w2 = k3 * Px + d * Nx;
    y[0] = l[2] * x[0] + w1;
#pragma unroll
    for (int i = 0; i < ND; i++) y[1 + i] = l[2] * x[1 + i] + v[i] * w1 + dscale(w2, nl[i]);
    y[NCU - 1] = l[2] * x[NCU - 1] + h * w1 + un * w2;
}

// The boundary flux fh[NCU] of fbou.m at one face point, from the interior state u, its gradient
// slots q, the trace uh and the boundary state ub = bcs(ib, :) (duals carry one derivative).
//   ns    (ns/fbou.m, fbou3d.m)  1 far field (an + An)(u - uh) - (an - An)(ub - uh), an = A_n(uh),
//         An = |A_n(uh)| (getan.m absolute 0 / 1); 2 adiabatic wall [u0 - uh0, -uh_m, fhat_E];
//         3 isothermal wall [u0 - uh0, -uh_m, gam gam1 Minf^2 uh_E/uh0 - ub_E]; 4 prescribed pressure,
//         the far-field form with ub replaced by [u0, u_m, p/gam1 + |u_m|^2/(2 u0)], p = (ub_E - 1/2) gam1;
//   euler (euler/fbou.m)  1, 3, 4 the same forms with the local Lax-Friedrichs scalars an = |un| + c
//         (eps > 0: ((|un| + c)^2/(eps c) + eps c)/2) and An = un - c of euler/getan.m at uh, p = ub_0
//         for 3; 2 slip wall u - (u_m . n) n - uh; 5 [u0, ub_m, u_E] - uh.
// Returns false for a type outside both lists.  Types 5 (ns: periodic = fhat) and 6 (Dirichlet)
// are handled by the caller.
template <int ND>
__device__ __noinline__ bool fbou_point(const FbouConst &fc, const PhysConst &pc, int ib, const double *ub,
                                        const double *nl, const D1 *u, const D1 *q, const D1 *uh, D1 *fh) {
    constexpr int NCU = ND + 2;
    const double gam1 = fc.gam - 1.0;
    D1 ui[NCU];
    const bool far = ib == 1 || ib == 4 || (fc.fam == 1 && ib == 3);
    if (far) {
        if (ib == 1) {
#pragma unroll
            for (int a = 0; a < NCU; a++) ui[a] = dc(ub[a]);
        } else {
            const double pb = (fc.fam == 1 && ib == 3) ? ub[0] : (ub[NCU - 1] - 0.5) * gam1;
            D1 ke = dc(0.0);
#pragma unroll
            for (int i = 0; i < ND; i++) {
                ui[1 + i] = u[1 + i];
                ke = ke + u[1 + i] * u[1 + i] / u[0];
            }
            ui[0] = u[0];
            ui[NCU - 1] = dc(pb / gam1) + dscale(ke, 0.5);
        }
        D1 a[NCU], b[NCU];
#pragma unroll
        for (int k = 0; k < NCU; k++) {
            a[k] = u[k] - ui[k];                        // (an + An)(u - uh) - (an - An)(ui - uh)
            b[k] = u[k] + ui[k] - dscale(uh[k], 2.0);   //   = an (u - ui) + An (u + ui - 2 uh)
        }
        if (fc.fam == 0) {
            D1 y[NCU];
            roe_apply<ND>(fc.gam, 0.0, nl, uh, false, a, fh);
            roe_apply<ND>(fc.gam, fc.eps, nl, uh, true, b, y);
#pragma unroll
            for (int k = 0; k < NCU; k++) fh[k] = fh[k] + y[k];
        } else {
            const D1 r = uh[0];
            D1 un = dc(0.0), af = dc(0.0);
#pragma unroll
            for (int i = 0; i < ND; i++) {
                const D1 vi = uh[1 + i] / r;
                un = un + dscale(vi, nl[i]);
                af = af + dscale(vi * vi, 0.5);
            }
            const D1 c = dsqrt(dscale(dscale(uh[NCU - 1] - r * af, gam1), fc.gam) / r);
            D1 an = dabs(un) + c;
            if (fc.eps > 0.0) {
                const D1 ec = dscale(c, fc.eps);
                an = dscale(an * an / ec + ec, 0.5);
            }
            const D1 An = un - c;
#pragma unroll
            for (int k = 0; k < NCU; k++) fh[k] = an * a[k] + An * b[k];
        }
        return true;
    }
    if (fc.fam == 0 && (ib == 2 || ib == 3)) {
        fh[0] = u[0] - uh[0];
#pragma unroll
        for (int i = 0; i < ND; i++) fh[1 + i] = dc(0.0) - uh[1 + i];
        if (ib == 3) {
            fh[NCU - 1] = dscale(uh[NCU - 1] / uh[0], fc.gam * gam1 * fc.m2) - dc(ub[NCU - 1]);
        } else {
            D1 f[NCU * ND];                                // the energy row of fhat at (uh, q)
            ns_flux<ND>(pc, uh, q, f);
            D1 e = dscale(u[NCU - 1] - uh[NCU - 1], pc.tau);
#pragma unroll
            for (int j = 0; j < ND; j++) e = e + dscale(f[(NCU - 1) + NCU * j], nl[j]);
            fh[NCU - 1] = e;
        }
        return true;
    }
    if (fc.fam == 1 && ib == 2) {
        D1 un = dc(0.0);
#pragma unroll
        for (int i = 0; i < ND; i++) un = un + dscale(u[1 + i], nl[i]);
        fh[0] = u[0] - uh[0];
#pragma unroll
        for (int i = 0; i < ND; i++) fh[1 + i] = u[1 + i] - dscale(un, nl[i]) - uh[1 + i];
        fh[NCU - 1] = u[NCU - 1] - uh[NCU - 1];
        return true;
    }
    if (fc.fam == 1 && ib == 5) {
#pragma unroll
        for (int a = 0; a < NCU; a++) fh[a] = ((a == 0 || a == NCU - 1) ? u[a] : dc(ub[a])) - uh[a];
        return true;
    }
    return false;
}

// --------------------------------------------------------------- block helpers
template <int NT>
__device__ __forceinline__ double block_reduce_max_abs(double v, double *red) {
    // not used on hot paths; kept simple
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double m = 0.0;
    for (int w = 0; w < NT / 32; w++) m = fmax(m, red[w]);
    __syncthreads();
    return m;
}

// In-place LU with partial pivoting of column-major A[n x n] (leading dimension lda) in
// shared memory by the whole block.  piv[k] = pivot row chosen at step k.  Returns
// nonzero (k+1) in *bad when a pivot is zero or not finite.  Warp 0 picks the pivot.
template <int NT>
__device__ void block_lu(double *A, int n, int lda, int *piv, int *bad) {
    for (int k = 0; k < n; k++) {
        if (threadIdx.x < 32) {
            double best = -1.0;
            int bi = k;
            for (int i = k + threadIdx.x; i < n; i += 32) {
                double v = fabs(A[i + lda * k]);
                if (v > best) { best = v; bi = i; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                double ob = __shfl_xor_sync(0xffffffffu, best, o);
                int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
            }
            if (threadIdx.x == 0) {
                piv[k] = bi;
                if (!(best > 0.0) || !isfinite(best)) { if (*bad == 0) *bad = k + 1; }
            }
        }
        __syncthreads();
        const int p = piv[k];
        if (p != k) {
            for (int j = threadIdx.x; j < n; j += NT) {
                double t = A[k + lda * j];
                A[k + lda * j] = A[p + lda * j];
                A[p + lda * j] = t;
            }
            __syncthreads();
        }
        const double akk = A[k + lda * k];
        const double inv = (akk != 0.0) ? 1.0 / akk : 0.0;
        for (int i = k + 1 + threadIdx.x; i < n; i += NT) A[i + lda * k] *= inv;
        __syncthreads();
        const int m = n - k - 1;
        for (int t = threadIdx.x; t < m * m; t += NT) {
            const int i = k + 1 + t % m, j = k + 1 + t / m;
            A[i + lda * j] -= A[i + lda * k] * A[k + lda * j];
        }
        __syncthreads();
    }
}

// Solve A X = B for ncols right-hand sides (columns of B, leading dimension ldb) with the
// factors of block_lu; one thread per column.
template <int NT>
__device__ void block_lu_solve(const double *LU, int n, int lda, const int *piv, double *B, int ldb, int ncols) {
    for (int c = threadIdx.x; c < ncols; c += NT) {
        double *b = B + (size_t)ldb * c;
        for (int k = 0; k < n; k++) {
            const int p = piv[k];
            if (p != k) { double t = b[k]; b[k] = b[p]; b[p] = t; }
        }
        for (int k = 0; k < n; k++) {
            const double bk = b[k];
            for (int i = k + 1; i < n; i++) b[i] -= LU[i + lda * k] * bk;
        }
        for (int k = n - 1; k >= 0; k--) {
            const double bk = b[k] / LU[k + lda * k];
            b[k] = bk;
            for (int i = 0; i < k; i++) b[i] -= LU[i + lda * k] * bk;
        }
    }
}


// Gauss-Jordan elimination with partial pivoting on the augmented system [A | B] held in
// shared memory (A: n x n, lda; B: n x nrhs, ldb), one __syncthreads per step.  The pivot
// search for step k+1 is fused into the step-k update: the threads that update column k+1
// of not-yet-pivoted rows post (|value| bits, row) into a 64-bit atomicMax slot (three
// rotating slots make one barrier per step sufficient).  Rows are never swapped; pivrow[k]
// records the physical row that carries unknown k.  On return B's row pivrow[k] holds the
// solution component k (already divided by the pivot).  *bad is set to k+1 when the pivot
// of step k is zero or not finite (the elimination still runs to completion).
// PIVOT = false eliminates in natural order (pivrow[k] = k), for SPD matrices such as M.
// Work per step: (n-1) rows x (n-k-1+nrhs) columns.
template <int NT, bool PIVOT = true>
__device__ void block_gauss_jordan(double *A, int lda, double *B, int ldb, int n, int nrhs,
                                   int *pivrow, int *rowused, unsigned long long *slot, int *bad) {
    const int tid = threadIdx.x;
    constexpr unsigned long long RMASK = 0x3FFull;   // rows < 1024
    for (int r = tid; r < n; r += NT) rowused[r] = 0;
    if (tid < 3) slot[tid] = 0ull;
    __syncthreads();
    // pivot for step 0
    for (int r = tid; r < n && PIVOT; r += NT) {
        const double v = fabs(A[r]);
        unsigned long long key = ((unsigned long long)__double_as_longlong(v) & ~RMASK) | (unsigned long long)r;
        atomicMax(&slot[0], key);
    }
    __syncthreads();
    for (int k = 0; k < n; k++) {
        const unsigned long long key = slot[k % 3];
        const int p = PIVOT ? (int)(key & RMASK) : k;
        const double piv = A[p + lda * k];
        if (tid == 0) {
            pivrow[k] = p;
            rowused[p] = 1;
            slot[(k + 2) % 3] = 0ull;
            if (!(fabs(piv) > 0.0) || !isfinite(piv)) { if (*bad == 0) *bad = k + 1; }
        }
        const double ipiv = (piv != 0.0) ? 1.0 / piv : 0.0;
        const int na = n - k - 1;             // remaining A columns k+1..n-1
        const int nc = na + nrhs;
        unsigned long long* nxt = &slot[(k + 1) % 3];
        for (int t = tid; t < n * nc; t += NT) {
            const int r = t % n, jj = t / n;
            if (r == p) continue;
            const double l = A[r + lda * k] * ipiv;
            if (jj < na) {
                const int j = k + 1 + jj;
                const double v = A[r + lda * j] - l * A[p + lda * j];
                A[r + lda * j] = v;
                if (PIVOT && jj == 0 && !rowused[r]) {
                    unsigned long long kk = ((unsigned long long)__double_as_longlong(fabs(v)) & ~RMASK) | (unsigned long long)r;
                    atomicMax(nxt, kk);
                }
            } else {
                const int j = jj - na;
                B[r + ldb * j] -= l * B[p + ldb * j];
            }
        }
        __syncthreads();
    }
    // scale: unknown k lives in row pivrow[k]
    for (int t = tid; t < n * nrhs; t += NT) {
        const int k = t % n, j = t / n;
        const int r = pivrow[k];
        B[r + ldb * j] /= A[r + lda * k];
    }
    __syncthreads();
}

// Gauss-Jordan elimination of the augmented system [A | B] (A: N x N, B: N x NR, both
// column-major with leading dimension N, in shared memory) with the matrix held in
// REGISTERS: thread (tr, tc) = (tid % TR, tid / TR) owns rows tr + i*TR and columns
// tc + jj*TC of the augmented matrix.  Per step k: the pivot row is broadcast inside each
// TR-lane group with __shfl_sync, the multipliers come from a shared copy of column k that
// the owners of column k wrote at the end of step k-1, and the owners also picked the
// step-k pivot there (max |value| over the rows not yet used, reduced with shuffles inside
// their TR-lane group), so one barrier per step suffices.  On return B holds the solution in natural row
// order.  PIVOT = false eliminates in natural order (SPD matrices).  *bad = k+1 for the
// first zero or non-finite pivot.  Shared scratch: pcol[2N] (column copy, double-buffered),
// diag[N], rowvar[N] (ints), slot[2] (ints).
template <typename T, int N, int NR1, int NR2, bool IDENT2, int NT, int TR, bool PIVOT>
__device__ __forceinline__ void gj_regs_t(const double *__restrict__ A, double *B, double *B2, T *pcol, T *diag,
                                          int *rowvar, int *slot, int *bad) {
    constexpr int NR = NR1 + NR2;
    static_assert(32 % TR == 0 && NT % TR == 0, "TR must divide 32 and NT");
    constexpr int NCOL = N + NR;
    constexpr int TC = NT / TR;
    constexpr int RPT = (N + TR - 1) / TR;
    constexpr int CPT = (NCOL + TC - 1) / TC;
    const int tid = threadIdx.x, tr = tid % TR, tc = tid / TR, lane = tid & 31;
    const unsigned gmask = (TR == 32) ? 0xffffffffu : (((1u << TR) - 1u) << (lane & ~(TR - 1)));
    T a[RPT][CPT];
#pragma unroll
    for (int i = 0; i < RPT; i++)
#pragma unroll
        for (int jj = 0; jj < CPT; jj++) {
            const int r = tr + i * TR, j = tc + jj * TC;
            double v = 0.0;
            if (r < N && j < NCOL) {
                if (j < N) v = A[r + N * j];
                else if (j < N + NR1) v = B[r + N * (j - N)];
                else v = IDENT2 ? ((j - N - NR1 == r) ? 1.0 : 0.0) : B2[r + N * (j - N - NR1)];
            }
            a[i][jj] = (T)v;
        }
    unsigned used = 0u;
    // owners of column kc publish it and choose its pivot row: key = bits of (float)|v| with
    // the low 10 bits replaced by the row (|v| within 2^-13 relative counts as a tie, won
    // by the higher row; NaN wins so that it is reported)
    auto publish = [&](int kc, int jq) {
        T *pn = pcol + (kc & 1) * N;
        unsigned best = 0u;
#pragma unroll
        for (int i = 0; i < RPT; i++) {
            const int r = tr + i * TR;
            T v = a[i][0];
#pragma unroll
            for (int jj = 1; jj < CPT; jj++) if (jq == jj) v = a[i][jj];
            if (r < N) {
                pn[r] = v;
                if (PIVOT && !((used >> i) & 1u)) {
                    const float av = (float)fabs(v);
                    const unsigned key = (av == av ? (__float_as_uint(av) & ~0x3FFu) : 0xFFFFFC00u) | (unsigned)r;
                    best = key > best ? key : best;
                }
            }
        }
        if (PIVOT) {
#pragma unroll
            for (int o = TR / 2; o > 0; o >>= 1) {
                const unsigned ob = __shfl_xor_sync(gmask, best, o, TR);
                best = ob > best ? ob : best;
            }
            if (tr == 0) slot[kc & 1] = (int)(best & 0x3FFu);
        }
    };
    if (tc == 0) publish(0, 0);
    __syncthreads();
    for (int k = 0; k < N; k++) {
        const int p = PIVOT ? slot[k & 1] : k;
        const T *pc = pcol + (k & 1) * N;
        const T piv = pc[p];
        const T ipiv = (piv != (T)0) ? (T)1 / piv : (T)0;
        if (tid == 0) {
            diag[k] = piv;
            rowvar[p] = k;
            if (!(fabs(piv) > 0.0) || !isfinite(piv)) { if (*bad == 0) *bad = k + 1; }
        }
        if (p % TR == tr) used |= 1u << (p / TR);
        T l[RPT];
#pragma unroll
        for (int i = 0; i < RPT; i++) {
            const int r = tr + i * TR;
            l[i] = (r < N && r != p) ? pc[r] * ipiv : (T)0;
        }
        const int src = (lane & ~(TR - 1)) | (p % TR);
        const int ip = p / TR;
#pragma unroll
        for (int jj = 0; jj < CPT; jj++) {
            T mine = a[0][jj];
#pragma unroll
            for (int i = 1; i < RPT; i++) if (ip == i) mine = a[i][jj];
            const T pv = __shfl_sync(0xffffffffu, mine, src);
            const int j = tc + jj * TC;
            if (j > k) {
#pragma unroll
                for (int i = 0; i < RPT; i++) a[i][jj] -= l[i] * pv;
            }
        }
        const int k1 = k + 1;
        if (k1 < N && tc == k1 % TC) publish(k1, k1 / TC);
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < RPT; i++)
#pragma unroll
        for (int jj = 0; jj < CPT; jj++) {
            const int r = tr + i * TR, j = tc + jj * TC;
            if (r < N && j >= N && j < NCOL) {
                const int var = rowvar[r];
                const double v = (double)(a[i][jj] / diag[var]);
                if (j < N + NR1) B[var + N * (j - N)] = v;
                else B2[var + N * (j - N - NR1)] = v;
            }
        }
    __syncthreads();
}
template <int N, int NR, int NT, int TR, bool PIVOT>
__device__ __forceinline__ void gj_regs(const double *__restrict__ A, double *B, double *pcol, double *diag,
                                        int *rowvar, int *slot, int *bad) {
    gj_regs_t<double, N, NR, 0, false, NT, TR, PIVOT>(A, B, nullptr, pcol, diag, rowvar, slot, bad);
}

// Unpivoted Gauss-Jordan on [A | B] with the matrix in registers (layout as gj_regs), the
// step loop fully unrolled so every pivot position is a compile-time constant.  The owner
// lane of the next pivot row publishes the next column and the reciprocal of the next
// pivot at the end of each step.  Used for M (symmetric positive definite) and as the
// fast path for the local matrix SD, whose result is then checked (backward error) and
// redone with gj_regs<..., PIVOT = true> when the check fails.  ROT > 0 eliminates the
// symmetrically permuted system (P A P^T) (P x) = P B with (P v)[i] = v[(i + ROT) % N]: for
// the local matrix SD with ROT = npv the density unknowns (component 0) come last, which
// removes the structurally zero density pivots of interior nodes (the continuity flux does
// not depend on the density).  Results are returned in natural order.  *bad = k+1 for the
// first zero or non-finite pivot.  Shared scratch: pcol[2N + 2].
template <typename T, int N, int NR1, int NR2, bool IDENT2, int NT, int TR, int ROT = 0>
__device__ __forceinline__ void gj_regs_nopiv_t(const double *__restrict__ A, double *B, double *B2, T *pcol, int *bad) {
    constexpr int NR = NR1 + NR2;
    static_assert(32 % TR == 0 && NT % TR == 0, "TR must divide 32 and NT");
    constexpr int NCOL = N + NR;
    constexpr int TC = NT / TR;
    constexpr int RPT = (N + TR - 1) / TR;
    constexpr int CPT = (NCOL + TC - 1) / TC;
    const int tid = threadIdx.x, tr = tid % TR, tc = tid / TR, lane = tid & 31;
    auto rot = [](int x) { return ROT == 0 ? x : (x + ROT < N ? x + ROT : x + ROT - N); };
    T a[RPT][CPT];
#pragma unroll
    for (int i = 0; i < RPT; i++)
#pragma unroll
        for (int jj = 0; jj < CPT; jj++) {
            const int r = tr + i * TR, j = tc + jj * TC;
            double v = 0.0;
            if (r < N && j < NCOL) {
                const int pr = rot(r);
                if (j < N) v = A[pr + N * rot(j)];
                else if (j < N + NR1) v = B[pr + N * (j - N)];
                else v = IDENT2 ? ((j - N - NR1 == pr) ? 1.0 : 0.0) : B2[pr + N * (j - N - NR1)];
            }
            a[i][jj] = (T)v;
        }
    // column 0 and 1/pivot_0
    if (tc == 0) {
#pragma unroll
        for (int i = 0; i < RPT; i++) {
            const int r = tr + i * TR;
            if (r < N) pcol[r] = a[i][0];
            if (r == 0) pcol[2 * N] = (T)1 / a[i][0];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; k++) {
        const T *pc = pcol + (k & 1) * N;
        const T ipiv = pcol[2 * N + (k & 1)];
        T l[RPT];
#pragma unroll
        for (int i = 0; i < RPT; i++) {
            const int r = tr + i * TR;
            l[i] = (r < N && r != k) ? pc[r] * ipiv : (T)0;
        }
        const int src = (lane & ~(TR - 1)) | (k % TR);
#pragma unroll
        for (int jj = 0; jj < CPT; jj++) {
            const T pv = __shfl_sync(0xffffffffu, a[k / TR][jj], src);
            if (tc + jj * TC > k) {
#pragma unroll
                for (int i = 0; i < RPT; i++) a[i][jj] -= l[i] * pv;
            }
        }
        if (k + 1 < N && tc == (k + 1) % TC) {
            T *pn = pcol + ((k + 1) & 1) * N;
#pragma unroll
            for (int i = 0; i < RPT; i++) {
                const int r = tr + i * TR;
                const T v = a[i][(k + 1) / TC];
                if (r < N) pn[r] = v;
                if (r == k + 1) {
                    if (!(fabs((double)v) > 0.0) || !isfinite((double)v)) { if (*bad == 0) *bad = k + 2; }
                    pcol[2 * N + ((k + 1) & 1)] = (v != (T)0) ? (T)1 / v : (T)0;
                }
            }
        }
        if (k == 0 && tid == 0) {
            const double v0 = (double)pc[0];
            if (!(fabs(v0) > 0.0) || !isfinite(v0)) { if (*bad == 0) *bad = 1; }
        }
        __syncthreads();
    }
    // unknown k lives in row k and is divided by that row's diagonal entry (the pivot)
#pragma unroll
    for (int i = 0; i < RPT; i++)
#pragma unroll
        for (int jj = 0; jj < CPT; jj++) {
            const int r = tr + i * TR, j = tc + jj * TC;
            if (r < N && j == r) pcol[r] = a[i][jj];
        }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < RPT; i++)
#pragma unroll
        for (int jj = 0; jj < CPT; jj++) {
            const int r = tr + i * TR, j = tc + jj * TC;
            if (r < N && j >= N && j < NCOL) {
                const double v = (double)(a[i][jj] / pcol[r]);
                const int pr = rot(r);
                if (j < N + NR1) B[pr + N * (j - N)] = v;
                else B2[pr + N * (j - N - NR1)] = v;
            }
        }
    __syncthreads();
}

template <int N, int NR, int NT, int TR, int ROT = 0>
__device__ __forceinline__ void gj_regs_nopiv(const double *__restrict__ A, double *B, double *pcol, int *bad) {
    gj_regs_nopiv_t<double, N, NR, 0, false, NT, TR, ROT>(A, B, nullptr, pcol, bad);
}

// Batched small GEMM with register tiles, spread over the NT threads of a CTA:
//   for b < NB, m < M, n < N:  store(b, m, n, sum_{k < K} a(b, m, k) * bb(b, k, n))
// Each thread owns TM x TN outputs of one batch entry, so every loaded value feeds TN (or
// TM) multiply-adds; a(...) / bb(...) return the operands (usually shared-memory reads) and
// store(...) consumes each result.  Threads are laid out m-tile fastest.  UK is the unroll
// factor of the k loop (K = fully unrolled: every k a compile-time constant).
template <int NB, int M, int N, int K, int TM, int TN, int NT, int UK = K, class FA, class FB, class FS>
__device__ __forceinline__ void tile_gemm(FA a, FB bb, FS store) {
    constexpr int MT = (M + TM - 1) / TM, NTL = (N + TN - 1) / TN;
    for (int t = threadIdx.x; t < NB * MT * NTL; t += NT) {
        const int mt = t % MT, nt = (t / MT) % NTL, b = t / (MT * NTL);
        const int m0 = mt * TM, n0 = nt * TN;
        double acc[TM][TN];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++) acc[i][j] = 0.0;
#pragma unroll UK
        for (int k = 0; k < K; k++) {
            double av[TM], bv[TN];
#pragma unroll
            for (int i = 0; i < TM; i++) av[i] = (M % TM == 0 || m0 + i < M) ? a(b, m0 + i, k) : 0.0;
#pragma unroll
            for (int j = 0; j < TN; j++) bv[j] = (N % TN == 0 || n0 + j < N) ? bb(b, k, n0 + j) : 0.0;
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int j = 0; j < TN; j++) acc[i][j] += av[i] * bv[j];
        }
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++)
                if ((M % TM == 0 || m0 + i < M) && (N % TN == 0 || n0 + j < N)) store(b, m0 + i, n0 + j, acc[i][j]);
    }
}

}  // namespace hdgx
