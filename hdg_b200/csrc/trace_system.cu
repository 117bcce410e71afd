// trace_system.cu -- the condensed (trace) system on the GPU, FP64.
//
//   gather_uh       kernel/hdg_assemble.m:34      UHe(:,:,e) = UH(:, elcon(:,e))
//   globalassembly  kernel/globalassembly.m:21-37 block-CSR Hg, Rg (atomics-free gather: every
//                   block / face row pulls its <= 2 element contributions)
//   matvec          kernel/matvec.m               y = Hg x
//   bilu0_factor    kernel/computeBILU0.m         block ILU(0) in a multicolour order:
//                   the rows of one colour share no block, so each colour is one launch
//                   with one CTA per row (left-looking form of the reference's
//                   right-looking update; identical factors for the same ordering)
//   bilu0_apply     kernel/applyBILU0.m           forward sweep by colour, backward sweep by
//                   colour in reverse, one warp per row
//   backsub         kernel/hdg_solve.m:119-121    DUDGT = DUDG + DUDG_DUH * DUH(elcon)
// Block storage: Hg[bs, bs, nnzb] column-major blocks, rowpts[nf+1] (int64 offsets),
// colind[nnzb] (1-based), diagonal block first in every row.
#include <cuda_runtime.h>
#include <math.h>
#include "hdgx_common.cuh"
#include "trace_internal.cuh"

namespace hdgx {

__global__ void gather_uh_kernel(int ncu, int ndf, int ne, const int *__restrict__ elcon,
                                 const double *__restrict__ UH, double *__restrict__ UHe) {
    const size_t n = (size_t)ncu * ndf * ne;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(t % ncu);
        const size_t fe = t / ncu;
        const int g = elcon[fe] - 1;
        UHe[t] = UH[c + (size_t)ncu * g];
    }
}

// Hg(:,:,k): block row i = face, block column j; contributions (e, a, b) listed per block
// (at most 2: the two elements of face i when j == i, else the one element holding both).
__global__ void assemble_h_kernel(int ncu, int npf, int nfe, long long nnzb, const int *__restrict__ blk_e,
                                  const int *__restrict__ blk_ab, const int *__restrict__ blk_row,
                                  const int *__restrict__ colind, const int *__restrict__ elcon,
                                  const double *__restrict__ AE, double *__restrict__ Hg) {
    const int bs = ncu * npf, ndf = npf * nfe, nh = ncu * ndf;
    for (long long k = blockIdx.x; k < nnzb; k += gridDim.x) {
        const int i = blk_row[k], j = colind[k] - 1;
        double *H = Hg + (size_t)bs * bs * k;
        for (int t = threadIdx.x; t < bs * bs; t += blockDim.x) {
            const int rr = t % bs, cc = t / bs;
            const int c = rr % ncu, mi = rr / ncu, cp = cc % ncu, mj = cc / ncu;
            double v = 0.0;
#pragma unroll
            for (int s = 0; s < 2; s++) {
                const int e = blk_e[2 * k + s];
                if (e < 0) continue;
                const int ab = blk_ab[2 * k + s], a = ab & 0xff, b = ab >> 8;
                const int *el = elcon + (size_t)ndf * e;
                int n = 0, np = 0;
                for (int q = 0; q < npf; q++) {
                    if (el[q + npf * a] - 1 - npf * i == mi) n = q;
                    if (el[q + npf * b] - 1 - npf * j == mj) np = q;
                }
                v += AE[(size_t)nh * nh * e + (c + ncu * (n + npf * a)) + (size_t)nh * (cp + ncu * (np + npf * b))];
            }
            H[t] = v;
        }
    }
}

__global__ void assemble_r_kernel(int ncu, int npf, int nfe, int nf, const int *__restrict__ face_e,
                                  const int *__restrict__ face_a, const int *__restrict__ elcon,
                                  const double *__restrict__ FE, double *__restrict__ Rg) {
    const int bs = ncu * npf, ndf = npf * nfe, nh = ncu * ndf;
    const size_t n = (size_t)bs * nf;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const int rr = (int)(t % bs), i = (int)(t / bs), c = rr % ncu, mi = rr / ncu;
        double v = 0.0;
        for (int s = 0; s < 2; s++) {
            const int e = face_e[2 * i + s];
            if (e < 0) continue;
            const int a = face_a[2 * i + s];
            const int *el = elcon + (size_t)ndf * e;
            int nn = 0;
            for (int q = 0; q < npf; q++)
                if (el[q + npf * a] - 1 - npf * i == mi) nn = q;
            v += FE[(size_t)nh * e + c + ncu * (nn + npf * a)];
        }
        Rg[t] = v;
    }
}

// y = Hg x, one warp per block row; lanes split the row's bs entries and block columns.
__global__ void bsr_matvec_kernel(int nf, int bs, const long long *__restrict__ rowpts,
                                  const int *__restrict__ colind, const double *__restrict__ Hg,
                                  const double *__restrict__ x, double *__restrict__ y) {
    const int lane = threadIdx.x & 31;
    const int warps = blockDim.x >> 5;
    for (int i = blockIdx.x * warps + (threadIdx.x >> 5); i < nf; i += gridDim.x * warps) {
        for (int r0 = 0; r0 < bs; r0 += 32) {
            const int r = r0 + lane;
            double acc = 0.0;
            if (r < bs) {
                for (long long k = rowpts[i]; k < rowpts[i + 1]; k++) {
                    const double *H = Hg + (size_t)bs * bs * k;
                    const double *xj = x + (size_t)bs * (colind[k] - 1);
                    for (int c = 0; c < bs; c++) acc += H[r + bs * c] * xj[c];
                }
                y[(size_t)bs * i + r] = acc;
            }
        }
    }
}

// ---------------------------------------------------------------- BILU(0)
// Factor the rows of one colour.  pos[row] = position of the row in the elimination order.
// Row i (one CTA): for its lower neighbours k in increasing pos:
//   A_ik <- A_ik inv(U_kk); A_ii -= A_ik U_ki; A_ij -= A_ik U_kj (j common, pos(j) > pos(k))
// then A_ii <- inv(A_ii).  (computeBILU0.m:16-44 applies the same updates from row k's side.)
template <int NT>
__global__ void __launch_bounds__(NT) bilu0_color_kernel(int bs, const int *__restrict__ rows, int nrows,
                                                         const long long *__restrict__ rowpts,
                                                         const int *__restrict__ colind,
                                                         const int *__restrict__ pos, double *Mg,
                                                         int *status) {
    extern __shared__ __align__(16) double sm[];
    const int b2 = bs * bs;
    double *Aii = sm, *L = sm + b2, *T = sm + 2 * b2;    // T: bs x 2bs augmented scratch
    int *lower = reinterpret_cast<int *>(sm + 4 * b2);    // up to 64 lower neighbours (block idx)
    int *nl = lower + 64;
    int *piv = nl + 1;                                    // bs <= 128
    int *rowused = piv + 128;
    unsigned long long *slot = reinterpret_cast<unsigned long long *>(sm + 4 * b2 + 200);
    int *bad = reinterpret_cast<int *>(slot + 4);
    const int tid = threadIdx.x;
    for (int q = blockIdx.x; q < nrows; q += gridDim.x) {
        const int i = rows[q];
        const long long k0 = rowpts[i], k1 = rowpts[i + 1];
        const int pi = pos[i];
        if (tid == 0) {
            int n = 0;
            for (long long k = k0 + 1; k < k1 && n < 64; k++)
                if (pos[colind[k] - 1] < pi) lower[n++] = (int)k;
            // insertion sort by pos of the column
            for (int a = 1; a < n; a++) {
                int v = lower[a], b = a - 1;
                while (b >= 0 && pos[colind[lower[b]] - 1] > pos[colind[v] - 1]) { lower[b + 1] = lower[b]; b--; }
                lower[b + 1] = v;
            }
            *nl = n;
            *bad = 0;
        }
        for (int t = tid; t < b2; t += NT) Aii[t] = Mg[(size_t)b2 * k0 + t];
        __syncthreads();
        const int n = *nl;
        for (int s = 0; s < n; s++) {
            const long long kik = lower[s];
            const int kr = colind[kik] - 1;                     // the lower row k
            const long long kkk = rowpts[kr];                    // its inverted diagonal
            // L = A_ik * inv(U_kk)
            for (int t = tid; t < b2; t += NT) {
                const int r = t % bs, c = t / bs;
                const double *A = Mg + (size_t)b2 * kik, *D = Mg + (size_t)b2 * kkk;
                double v = 0.0;
                for (int m = 0; m < bs; m++) v += A[r + bs * m] * D[m + bs * c];
                L[t] = v;
            }
            __syncthreads();
            for (int t = tid; t < b2; t += NT) Mg[(size_t)b2 * kik + t] = L[t];
            // A_ii -= L U_ki ; A_ij -= L U_kj for the other blocks of row i
            for (long long kk = rowpts[kr] + 1; kk < rowpts[kr + 1]; kk++) {
                const int j = colind[kk] - 1;
                if (pos[j] <= pos[kr]) continue;                 // only the U part of row k
                long long kij = -1;
                if (j == i) kij = k0;
                else
                    for (long long k = k0 + 1; k < k1; k++) if (colind[k] - 1 == j) { kij = k; break; }
                if (kij < 0) continue;                           // no fill (ILU(0))
                const double *U = Mg + (size_t)b2 * kk;
                if (kij == k0) {
                    for (int t = tid; t < b2; t += NT) {
                        const int r = t % bs, c = t / bs;
                        double v = 0.0;
                        for (int m = 0; m < bs; m++) v += L[r + bs * m] * U[m + bs * c];
                        Aii[t] -= v;
                    }
                } else {
                    double *A = Mg + (size_t)b2 * kij;
                    for (int t = tid; t < b2; t += NT) {
                        const int r = t % bs, c = t / bs;
                        double v = 0.0;
                        for (int m = 0; m < bs; m++) v += L[r + bs * m] * U[m + bs * c];
                        A[t] -= v;
                    }
                }
                __syncthreads();
            }
            __syncthreads();
        }
        // invert A_ii: Gauss-Jordan on [A_ii | I]
        for (int t = tid; t < b2; t += NT) { T[t] = Aii[t]; T[b2 + t] = ((t % bs) == (t / bs)) ? 1.0 : 0.0; }
        __syncthreads();
        block_gauss_jordan<NT, true>(T, bs, T + b2, bs, bs, bs, piv, rowused, slot, bad);
        for (int t = tid; t < b2; t += NT) {
            const int r = t % bs, c = t / bs;
            Mg[(size_t)b2 * k0 + t] = T[b2 + piv[r] + bs * c];
        }
        if (tid == 0 && *bad && status) status[i] = 1;
        __syncthreads();
    }
}

// Forward sweep for the rows of one colour: y_i = x_i - sum_{pos(k) < pos(i)} L_ik y_k.
__global__ void bilu0_fwd_kernel(int bs, const int *__restrict__ rows, int nrows, const long long *__restrict__ rowpts,
                                 const int *__restrict__ colind, const int *__restrict__ pos,
                                 const double *__restrict__ Mg, const double *__restrict__ x, double *y) {
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (int q = blockIdx.x * warps + (threadIdx.x >> 5); q < nrows; q += gridDim.x * warps) {
        const int i = rows[q], pi = pos[i];
        for (int r0 = 0; r0 < bs; r0 += 32) {
            const int r = r0 + lane;
            if (r >= bs) continue;
            double acc = x[(size_t)bs * i + r];
            for (long long k = rowpts[i] + 1; k < rowpts[i + 1]; k++) {
                const int j = colind[k] - 1;
                if (pos[j] >= pi) continue;
                const double *Lk = Mg + (size_t)bs * bs * k, *yj = y + (size_t)bs * j;
                for (int c = 0; c < bs; c++) acc -= Lk[r + bs * c] * yj[c];
            }
            y[(size_t)bs * i + r] = acc;
        }
    }
}

// Backward sweep for the rows of one colour: v_i = inv(U_ii) (y_i - sum_{pos(j) > pos(i)} U_ij v_j).
__global__ void bilu0_bwd_kernel(int bs, const int *__restrict__ rows, int nrows, const long long *__restrict__ rowpts,
                                 const int *__restrict__ colind, const int *__restrict__ pos,
                                 const double *__restrict__ Mg, const double *__restrict__ y, double *v) {
    extern __shared__ double sh[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, warps = blockDim.x >> 5;
    double *t = sh + w * bs;
    for (int q = blockIdx.x * warps + w; q < nrows; q += gridDim.x * warps) {
        const int i = rows[q], pi = pos[i];
        for (int r = lane; r < bs; r += 32) {
            double acc = y[(size_t)bs * i + r];
            for (long long k = rowpts[i] + 1; k < rowpts[i + 1]; k++) {
                const int j = colind[k] - 1;
                if (pos[j] <= pi) continue;
                const double *U = Mg + (size_t)bs * bs * k, *vj = v + (size_t)bs * j;
                for (int c = 0; c < bs; c++) acc -= U[r + bs * c] * vj[c];
            }
            t[r] = acc;
        }
        __syncwarp();
        const double *D = Mg + (size_t)bs * bs * rowpts[i];
        for (int r = lane; r < bs; r += 32) {
            double s = 0.0;
            for (int c = 0; c < bs; c++) s += D[r + bs * c] * t[c];
            v[(size_t)bs * i + r] = s;
        }
        __syncwarp();
    }
}

// DUDGT = DUDG + DUDG_DUH * DUH(elcon): one CTA per element, the element's trace update
// gathered into shared memory.
__global__ void backsub_kernel(int ne, int nq, int ncu, int ndf, const int *__restrict__ elcon,
                               const double *__restrict__ DUDG, const double *__restrict__ DUDG_DUH,
                               const double *__restrict__ DUH, double *__restrict__ out) {
    extern __shared__ double u[];
    const int nh = ncu * ndf;
    for (int e = blockIdx.x; e < ne; e += gridDim.x) {
        for (int k = threadIdx.x; k < nh; k += blockDim.x) {
            const int c = k % ncu, f = k / ncu;
            u[k] = DUH[c + (size_t)ncu * (elcon[(size_t)ndf * e + f] - 1)];
        }
        __syncthreads();
        const double *D = DUDG_DUH + (size_t)nq * nh * e;
        for (int q = threadIdx.x; q < nq; q += blockDim.x) {
            double s = DUDG[(size_t)nq * e + q];
            for (int k = 0; k < nh; k++) s += D[q + (size_t)nq * k] * u[k];
            out[(size_t)nq * e + q] = s;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ vector kernels
// Deterministic dot product: per-block partial sums, then one block sums them in order.
__global__ void dot_partial_kernel(size_t n, const double *__restrict__ a, const double *__restrict__ b, double *part) {
    __shared__ double red[32];
    double s = 0.0;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        s += a[t] * b[t];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) part[blockIdx.x] = s;
    }
}

// out = sum(part[0:np]) (sqrt when do_sqrt); also out2 = -out when out2 != nullptr.
__global__ void dot_final_kernel(int np, const double *part, double *out, int do_sqrt) {
    __shared__ double red[32];
    double s = 0.0;
    for (int t = threadIdx.x; t < np; t += blockDim.x) s += part[t];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) r += red[w];
        *out = do_sqrt ? sqrt(r) : r;
    }
}

// y += alpha * x where alpha = sgn * (*palpha) (device scalar) or the host value when palpha == nullptr.
__global__ void axpy_kernel(size_t n, const double *palpha, double sgn, const double *__restrict__ x, double *y) {
    const double a = sgn * (*palpha);
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        y[t] += a * x[t];
}

// y = x / (*pnorm)
__global__ void scale_div_kernel(size_t n, const double *pnorm, const double *__restrict__ x, double *y) {
    const double d = *pnorm;
    const double s = (d != 0.0) ? 1.0 / d : 0.0;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        y[t] = x[t] * s;
}

// z = x - y
__global__ void sub_kernel(size_t n, const double *__restrict__ x, const double *__restrict__ y, double *z) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        z[t] = x[t] - y[t];
}

// y = a*x + b*y (host scalars)
__global__ void axpby_kernel(size_t n, double a, const double *__restrict__ x, double b, double *y) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        y[t] = a * x[t] + b * y[t];
}

// GMRES state on the device: H[(m+1) x m] column-major, cs, sn, g[m+1], scalars.

// Apply the previous rotations to column j of H, form the new one, update g.  One thread.
__global__ void givens_kernel(GmresState s, int m, int j) {
    double *h = s.H + (size_t)(m + 1) * j;
    for (int i = 0; i < j; i++) {
        const double a = h[i], b = h[i + 1];
        h[i] = s.cs[i] * a + s.sn[i] * b;
        h[i + 1] = -s.sn[i] * a + s.cs[i] * b;
    }
    const double a = h[j], b = h[j + 1];
    const double den = sqrt(a * a + b * b);
    const double c = (den != 0.0) ? a / den : 1.0, sn = (den != 0.0) ? b / den : 0.0;
    s.cs[j] = c; s.sn[j] = sn;
    h[j] = den; h[j + 1] = 0.0;
    s.g[j + 1] = -sn * s.g[j];
    s.g[j] = c * s.g[j];
    s.scal[1] = fabs(s.g[j + 1]);
    if (s.hist) s.hist[j] = s.scal[1];
}

// Back substitution of the triangular Hessenberg system for y[0:k].  One thread.
__global__ void hess_solve_kernel(GmresState s, int m, int k) {
    for (int i = k - 1; i >= 0; i--) {
        double v = s.g[i];
        for (int l = i + 1; l < k; l++) v -= s.H[i + (size_t)(m + 1) * l] * s.y[l];
        s.y[i] = v / s.H[i + (size_t)(m + 1) * i];
    }
}

// g = [beta, 0, ...]
__global__ void gmres_init_kernel(GmresState s, int m) {
    for (int i = threadIdx.x; i <= m; i += blockDim.x) s.g[i] = (i == 0) ? s.scal[0] : 0.0;
}

}  // namespace hdgx

namespace hdgx {
template __global__ void bilu0_color_kernel<256>(int, const int *, int, const long long *, const int *, const int *,
                                                 double *, int *);
}

// ===================================================================== MDF-ordered BILU(0)
// computeMDFordering.m: C(k) = || inv(H_ii) H_ik ||_F for every block of row i.  One CTA per
// row: Gauss-Jordan on [H_ii | H_i,row] (the row's blocks are contiguous in Hg).
namespace hdgx {
template <int NT>
__global__ void __launch_bounds__(NT) block_norms_kernel(int bs, int nf, const long long *__restrict__ rowpts,
                                                         const double *__restrict__ Hg, double *__restrict__ C) {
    extern __shared__ __align__(16) double sm[];
    const int b2 = bs * bs;
    double *A = sm, *Inv = sm + b2;                       // [H_ii | I] -> inv(H_ii)
    int *piv = reinterpret_cast<int *>(sm + 2 * b2);
    int *rowused = piv + 128;
    unsigned long long *slot = reinterpret_cast<unsigned long long *>(sm + 2 * b2 + 130);
    int *bad = reinterpret_cast<int *>(slot + 4);
    for (int i = blockIdx.x; i < nf; i += gridDim.x) {
        const long long k0 = rowpts[i], k1 = rowpts[i + 1];
        const double *H = Hg + (size_t)b2 * k0;
        for (int t = threadIdx.x; t < b2; t += NT) { A[t] = H[t]; Inv[t] = ((t % bs) == (t / bs)) ? 1.0 : 0.0; }
        if (threadIdx.x == 0) *bad = 0;
        __syncthreads();
        block_gauss_jordan<NT, true>(A, bs, Inv, bs, bs, bs, piv, rowused, slot, bad);
        // row r of inv(H_ii) is in Inv row piv[r]; || inv(H_ii) H_ik ||_F, one warp per block
        for (long long k = k0 + (threadIdx.x >> 5); k < k1; k += NT / 32) {
            const double *B = Hg + (size_t)b2 * k;
            double s = 0.0;
            for (int t = threadIdx.x & 31; t < b2; t += 32) {
                const int r = t % bs, c = t / bs;
                double v = 0.0;
                for (int m = 0; m < bs; m++) v += Inv[piv[r] + bs * m] * B[m + bs * c];
                s += v * v;
            }
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if ((threadIdx.x & 31) == 0) C[k] = sqrt(s);
        }
        __syncthreads();
    }
}
template __global__ void block_norms_kernel<256>(int, int, const long long *, const double *, double *);

// Flag-scheduled sweeps and factorisation in an arbitrary sequential order.  sched[] layout:
// [0] epoch, [1] work counter, [2] error flag, [3] poll limit of every wait (0: HDGX_SPIN_LIMIT),
// [4 + i] ready flag of row i.  Rows are taken in order through the counter, so a row only waits
// for rows taken before it by CTAs / warps that are already running; every wait is bounded,
// after which the error flag is raised and the row proceeds.
#define HDGX_SPIN_LIMIT (1 << 22)

__device__ __forceinline__ int poll_limit(const int *sched) {
    const int l = sched[3];
    return l > 0 ? l : HDGX_SPIN_LIMIT;
}

// ------------------------------------------------------------- fused Gram-Schmidt step
// Blocks of one cooperative launch meet here.  Thread 0 of each block arrives on a counter; the
// last one resets it and advances the generation; the others poll the generation with a bounded
// wait (after HDGX_SPIN_LIMIT polls the error flag is raised and the block goes on).
__device__ __forceinline__ void grid_barrier(unsigned *bar, unsigned nblocks, int *err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == nblocks - 1) {
            bar[0] = 0;
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            int n = 0;
            while (*gen == g) {
                if (++n > HDGX_SPIN_LIMIT) { atomicExch(err, 1); break; }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// One Arnoldi orthogonalisation of GMRES (modified Gram-Schmidt, gmres_bilu0.m:59-63: for
// i < nv, h_i = v_i . w, w -= h_i v_i; then h_nv = |w|, w /= h_nv) as ONE cooperative launch
// instead of 3 (nv + 1) small ones.  The grid is that of the two-pass dot product it replaces,
// each block forms its partial sums over the same grid-stride elements and every block adds the
// partials in the order of dot_final_kernel (256 threads), so the results are the same bit for
// bit; every element of w is read and written by the same thread throughout, so one grid
// barrier per product suffices (partials alternate between two halves of part[2 * grid]).
__global__ void __launch_bounds__(256) mgs_coop_kernel(size_t n, int nv, const double *__restrict__ V, double *w,
                                                       double *hcol, double *part, unsigned *bar, int *err) {
    __shared__ double red[32];
    __shared__ double hval;
    const unsigned G = gridDim.x;
    const int tid = threadIdx.x;
    for (int i = 0; i <= nv; i++) {
        const double *a = i < nv ? V + n * i : w;
        double *pp = part + (size_t)(i & 1) * G;
        double s = 0.0;
        for (size_t t = blockIdx.x * (size_t)blockDim.x + tid; t < n; t += (size_t)G * blockDim.x) s += a[t] * w[t];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((tid & 31) == 0) red[tid >> 5] = s;
        __syncthreads();
        if (tid < 32) {
            s = (tid < (int)(blockDim.x >> 5)) ? red[tid] : 0.0;
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (tid == 0) pp[blockIdx.x] = s;
        }
        grid_barrier(bar, G, err);
        s = 0.0;
        for (int t = tid; t < (int)G; t += blockDim.x) s += __ldcg(pp + t);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((tid & 31) == 0) red[tid >> 5] = s;
        __syncthreads();
        if (tid == 0) {
            double r = 0.0;
            for (int q = 0; q < (int)(blockDim.x >> 5); q++) r += red[q];
            hval = (i < nv) ? r : sqrt(r);
            if (blockIdx.x == 0) hcol[i] = hval;
        }
        __syncthreads();
        const double h = hval;
        if (i < nv) {
            const double al = -1.0 * h;
            for (size_t t = blockIdx.x * (size_t)blockDim.x + tid; t < n; t += (size_t)G * blockDim.x) w[t] += al * a[t];
        } else {
            const double sc = (h != 0.0) ? 1.0 / h : 0.0;
            for (size_t t = blockIdx.x * (size_t)blockDim.x + tid; t < n; t += (size_t)G * blockDim.x) w[t] = w[t] * sc;
        }
        __syncthreads();
    }
}

__device__ __forceinline__ int load_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void wait_flag(const int *flag, int epoch, int *err, int limit) {
    int n = 0;
    while (load_acquire(flag) != epoch) {
        if (++n > limit) { atomicExch(err, 1); break; }
        if (n > 64) __nanosleep(64);
    }
}

__global__ void sched_begin_kernel(int *sched) {
    sched[0] += 1;      // new epoch: every flag now reads "not ready"
    sched[1] = 0;
}

template <int NT>
__global__ void __launch_bounds__(NT) bilu0_sched_factor_kernel(int bs, int nf, const int *__restrict__ order,
                                                                const long long *__restrict__ rowpts,
                                                                const int *__restrict__ colind,
                                                                const int *__restrict__ pos, double *Mg,
                                                                int *sched, int *status) {
    extern __shared__ __align__(16) double sm[];
    const int b2 = bs * bs;
    double *Aii = sm, *L = sm + b2, *T = sm + 2 * b2;
    int *lower = reinterpret_cast<int *>(sm + 4 * b2);
    int *nl = lower + 64;
    int *piv = nl + 1;
    int *rowused = piv + 128;
    int *cur = rowused + 128;
    unsigned long long *slot = reinterpret_cast<unsigned long long *>(sm + 4 * b2 + 200);
    int *bad = reinterpret_cast<int *>(slot + 4);
    const int tid = threadIdx.x;
    const int epoch = sched[0], limit = poll_limit(sched);
    int *flags = sched + 4, *err = sched + 2;
    for (;;) {
        if (tid == 0) {
            const int q = atomicAdd(&sched[1], 1);
            *cur = q < nf ? order[q] : -1;
        }
        __syncthreads();
        const int i = *cur;
        if (i < 0) break;
        const long long k0 = rowpts[i], k1 = rowpts[i + 1];
        const int pi = pos[i];
        if (tid == 0) {
            int n = 0;
            for (long long k = k0 + 1; k < k1 && n < 64; k++)
                if (pos[colind[k] - 1] < pi) lower[n++] = (int)k;
            for (int a = 1; a < n; a++) {
                int v = lower[a], b = a - 1;
                while (b >= 0 && pos[colind[lower[b]] - 1] > pos[colind[v] - 1]) { lower[b + 1] = lower[b]; b--; }
                lower[b + 1] = v;
            }
            *nl = n;
            *bad = 0;
            for (int s = 0; s < n; s++) wait_flag(flags + (colind[lower[s]] - 1), epoch, err, limit);
        }
        __syncthreads();
        for (int t = tid; t < b2; t += NT) Aii[t] = Mg[(size_t)b2 * k0 + t];
        __syncthreads();
        const int n = *nl;
        for (int s = 0; s < n; s++) {
            const long long kik = lower[s];
            const int kr = colind[kik] - 1;
            const long long kkk = rowpts[kr];
            for (int t = tid; t < b2; t += NT) {
                const int r = t % bs, c = t / bs;
                const double *A = Mg + (size_t)b2 * kik, *D = Mg + (size_t)b2 * kkk;
                double v = 0.0;
                for (int m = 0; m < bs; m++) v += A[r + bs * m] * __ldcg(D + m + bs * c);
                L[t] = v;
            }
            __syncthreads();
            for (int t = tid; t < b2; t += NT) Mg[(size_t)b2 * kik + t] = L[t];
            for (long long kk = rowpts[kr] + 1; kk < rowpts[kr + 1]; kk++) {
                const int j = colind[kk] - 1;
                if (pos[j] <= pos[kr]) continue;
                long long kij = -1;
                if (j == i) kij = k0;
                else
                    for (long long k = k0 + 1; k < k1; k++) if (colind[k] - 1 == j) { kij = k; break; }
                if (kij < 0) continue;
                const double *U = Mg + (size_t)b2 * kk;
                double *dst = (kij == k0) ? Aii : Mg + (size_t)b2 * kij;
                for (int t = tid; t < b2; t += NT) {
                    const int r = t % bs, c = t / bs;
                    double v = 0.0;
                    for (int m = 0; m < bs; m++) v += L[r + bs * m] * __ldcg(U + m + bs * c);
                    dst[t] -= v;
                }
                __syncthreads();
            }
            __syncthreads();
        }
        for (int t = tid; t < b2; t += NT) { T[t] = Aii[t]; T[b2 + t] = ((t % bs) == (t / bs)) ? 1.0 : 0.0; }
        __syncthreads();
        block_gauss_jordan<NT, true>(T, bs, T + b2, bs, bs, bs, piv, rowused, slot, bad);
        for (int t = tid; t < b2; t += NT) {
            const int r = t % bs, c = t / bs;
            Mg[(size_t)b2 * k0 + t] = T[b2 + piv[r] + bs * c];
        }
        if (tid == 0 && *bad && status) status[i] = 1;
        __threadfence();
        __syncthreads();
        if (tid == 0) atomicExch(flags + i, epoch);
    }
}
template __global__ void bilu0_sched_factor_kernel<256>(int, int, const int *, const long long *, const int *,
                                                        const int *, double *, int *, int *);

// Forward (dir = 0, order ascending, y = x - L y) or backward (dir = 1, order descending,
// v = inv(U_ii)(y - U v)) sweep, one warp per row.
__global__ void bilu0_sched_sweep_kernel(int bs, int nf, int dir, const int *__restrict__ order,
                                         const long long *__restrict__ rowpts, const int *__restrict__ colind,
                                         const int *__restrict__ pos, const double *__restrict__ Mg,
                                         const double *__restrict__ in, double *out, int *sched) {
    extern __shared__ double sh[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double *t = sh + w * bs;
    const int epoch = sched[0], limit = poll_limit(sched);
    int *flags = sched + 4, *err = sched + 2;
    for (;;) {
        int q = 0;
        if (lane == 0) q = atomicAdd(&sched[1], 1);
        q = __shfl_sync(0xffffffffu, q, 0);
        if (q >= nf) break;
        const int i = order[dir ? nf - 1 - q : q], pi = pos[i];
        const long long k0 = rowpts[i], k1 = rowpts[i + 1];
        if (lane == 0)
            for (long long k = k0 + 1; k < k1; k++) {
                const int j = colind[k] - 1;
                if (dir ? (pos[j] > pi) : (pos[j] < pi)) wait_flag(flags + j, epoch, err, limit);
            }
        __syncwarp();
        for (int r = lane; r < bs; r += 32) {
            double acc = in[(size_t)bs * i + r];
            for (long long k = k0 + 1; k < k1; k++) {
                const int j = colind[k] - 1;
                if (dir ? (pos[j] <= pi) : (pos[j] >= pi)) continue;
                const double *B = Mg + (size_t)bs * bs * k, *oj = out + (size_t)bs * j;
                for (int c = 0; c < bs; c++) acc -= B[r + bs * c] * __ldcg(oj + c);
            }
            t[r] = acc;
        }
        __syncwarp();
        for (int r = lane; r < bs; r += 32) {
            double v = t[r];
            if (dir) {
                const double *D = Mg + (size_t)bs * bs * k0;
                v = 0.0;
                for (int c = 0; c < bs; c++) v += D[r + bs * c] * t[c];
            }
            out[(size_t)bs * i + r] = v;
        }
        __syncwarp();
        if (lane == 0) {
            __threadfence();
            atomicExch(flags + i, epoch);
        }
    }
}
}  // namespace hdgx

// ------------------------------------------------------------------------------------------
// Block-size-specialised sweeps and matvec (BS known at compile time: every load of a block
// row is issued before the first multiply-add, so one memory latency covers a whole block).
namespace hdgx {
template <int BS>
__global__ void bilu0_fwd_bs_kernel(const int *__restrict__ rows, int nrows, const long long *__restrict__ rowpts,
                                    const int *__restrict__ colind, const int *__restrict__ pos,
                                    const double *__restrict__ Mg, const double *__restrict__ x, double *y) {
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (int q = blockIdx.x * warps + (threadIdx.x >> 5); q < nrows; q += gridDim.x * warps) {
        const int i = rows[q], pi = pos[i];
        for (int r = lane; r < BS; r += 32) {
            double acc = x[(size_t)BS * i + r];
            for (long long k = rowpts[i] + 1; k < rowpts[i + 1]; k++) {
                const int j = colind[k] - 1;
                if (pos[j] >= pi) continue;
                const double *Lk = Mg + (size_t)BS * BS * k, *yj = y + (size_t)BS * j;
                double lv[BS], yv[BS];
#pragma unroll
                for (int c = 0; c < BS; c++) { lv[c] = Lk[r + BS * c]; yv[c] = __ldcg(yj + c); }
#pragma unroll
                for (int c = 0; c < BS; c++) acc -= lv[c] * yv[c];
            }
            y[(size_t)BS * i + r] = acc;
        }
    }
}

template <int BS>
__global__ void bilu0_bwd_bs_kernel(const int *__restrict__ rows, int nrows, const long long *__restrict__ rowpts,
                                    const int *__restrict__ colind, const int *__restrict__ pos,
                                    const double *__restrict__ Mg, const double *__restrict__ y, double *v) {
    __shared__ double tsh[8][BS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, warps = blockDim.x >> 5;
    for (int q = blockIdx.x * warps + w; q < nrows; q += gridDim.x * warps) {
        const int i = rows[q], pi = pos[i];
        for (int r = lane; r < BS; r += 32) {
            double acc = y[(size_t)BS * i + r];
            for (long long k = rowpts[i] + 1; k < rowpts[i + 1]; k++) {
                const int j = colind[k] - 1;
                if (pos[j] <= pi) continue;
                const double *U = Mg + (size_t)BS * BS * k, *vj = v + (size_t)BS * j;
                double uv[BS], vv[BS];
#pragma unroll
                for (int c = 0; c < BS; c++) { uv[c] = U[r + BS * c]; vv[c] = __ldcg(vj + c); }
#pragma unroll
                for (int c = 0; c < BS; c++) acc -= uv[c] * vv[c];
            }
            tsh[w][r] = acc;
        }
        __syncwarp();
        const double *D = Mg + (size_t)BS * BS * rowpts[i];
        for (int r = lane; r < BS; r += 32) {
            double dv[BS];
#pragma unroll
            for (int c = 0; c < BS; c++) dv[c] = D[r + BS * c];
            double s = 0.0;
#pragma unroll
            for (int c = 0; c < BS; c++) s += dv[c] * tsh[w][c];
            v[(size_t)BS * i + r] = s;
        }
        __syncwarp();
    }
}

template <int BS>
__global__ void bsr_matvec_bs_kernel(int nf, const long long *__restrict__ rowpts, const int *__restrict__ colind,
                                     const double *__restrict__ Hg, const double *__restrict__ x,
                                     double *__restrict__ y) {
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (int i = blockIdx.x * warps + (threadIdx.x >> 5); i < nf; i += gridDim.x * warps) {
        for (int r = lane; r < BS; r += 32) {
            double acc = 0.0;
            for (long long k = rowpts[i]; k < rowpts[i + 1]; k++) {
                const double *H = Hg + (size_t)BS * BS * k, *xj = x + (size_t)BS * (colind[k] - 1);
                double hv[BS], xv[BS];
#pragma unroll
                for (int c = 0; c < BS; c++) { hv[c] = H[r + BS * c]; xv[c] = xj[c]; }
#pragma unroll
                for (int c = 0; c < BS; c++) acc += hv[c] * xv[c];
            }
            y[(size_t)BS * i + r] = acc;
        }
    }
}

#define HDGX_BS_LIST(X) X(8) X(12) X(15) X(16) X(20) X(30)
#define HDGX_INST(B)                                                                                             \
    template __global__ void bilu0_fwd_bs_kernel<B>(const int *, int, const long long *, const int *, const int *, \
                                                    const double *, const double *, double *);                     \
    template __global__ void bilu0_bwd_bs_kernel<B>(const int *, int, const long long *, const int *, const int *, \
                                                    const double *, const double *, double *);                     \
    template __global__ void bsr_matvec_bs_kernel<B>(int, const long long *, const int *, const double *,           \
                                                     const double *, double *);
HDGX_BS_LIST(HDGX_INST)
#undef HDGX_INST
}  // namespace hdgx
