// dense_block.cu -- the reference's dense face-block solver path (app.denseblock = 1):
//   kernel/arraymul.c:11-96          batched GEMM / GEMV                 -> hdgx_arraymul
//   kernel/mkDenseBlockSystem.m:9-95 block-Jacobi-scaled face blocks      -> hdgx_dense_block_system
//   kernel/gmres.m:1-111             GMRES(restart) on x + K gather(x)    -> hdgx_gmres_dense
//
// Face i's block row of the condensed matrix (diagonal block D_i, neighbour blocks H_ij for
// the faces j listed in f2f(2:end, i), mesh/mkmesh/mkf2f.m) is scaled by inv(D_i):
//   K(:, :, k, i) = inv(D_i) H_{i, f2f(k+1, i)},   F(:, i) = inv(D_i) R_i,
// here by solving D_i [F_i | K_i] = [R_i | H_i] (Gauss-Jordan with partial pivoting) rather
// than forming inv(D_i) first.  The GMRES operator is A x = x + K gather(x), unpreconditioned,
// with classical Gram-Schmidt in block form (gmres.m:80-81) and the Hessenberg least-squares
// problem solved by Givens rotations (the same minimiser as gmres.m:90's backslash).
#include <cuda_runtime.h>
#include <math.h>
#include "hdgx_common.cuh"
#include "trace_internal.cuh"

namespace hdgx {

// C(:, i) = A(:, :, i) B(:, i)   (arraymul.c:60-69); one thread per output row
__global__ void batched_gemv_kernel(int rows, int cols, int nb, const double *__restrict__ A,
                                    const double *__restrict__ B, double *__restrict__ C) {
    const size_t total = (size_t)rows * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(t % rows);
        const size_t i = t / rows;
        const double *a = A + (size_t)rows * cols * i + r, *b = B + (size_t)cols * i;
        double s = 0.0;
        for (int c = 0; c < cols; c++) s += a[(size_t)rows * c] * b[c];
        C[t] = s;
    }
}

// C(:, :, i) = A(:, :, i) B(:, :, i)   (arraymul.c:78-92); one thread per output entry
__global__ void batched_gemm_kernel(int rows, int inner, int cols, int nb, const double *__restrict__ A,
                                    const double *__restrict__ B, double *__restrict__ C) {
    const size_t total = (size_t)rows * cols * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(t % rows);
        const size_t ci = t / rows;
        const int c = (int)(ci % cols);
        const size_t i = ci / cols;
        const double *a = A + (size_t)rows * inner * i + r, *b = B + (size_t)inner * (c + (size_t)cols * i);
        double s = 0.0;
        for (int k = 0; k < inner; k++) s += a[(size_t)rows * k] * b[k];
        C[t] = s;
    }
}

// One CTA per face: D_i [F_i | K_i] = [R_i | H_i,f2f(2:end,i)]  (mkDenseBlockSystem.m:31-94)
template <int NT>
__global__ void __launch_bounds__(NT) dense_block_kernel(int bs, int nf, int nbf, const long long *__restrict__ rowpts,
                                                         const int *__restrict__ colind, const double *__restrict__ Hg,
                                                         const double *__restrict__ Rg, const int *__restrict__ f2f,
                                                         double *__restrict__ K, double *__restrict__ F, int *status) {
    extern __shared__ __align__(16) double sm[];
    const int nn = nbf - 1, nrhs = 1 + bs * nn, b2 = bs * bs;
    double *D = sm, *X = sm + b2;
    int *pivrow = reinterpret_cast<int *>(X + (size_t)bs * nrhs);
    int *rowused = pivrow + bs;
    int *src = rowused + bs;                               // [nn] block index of each neighbour, or -1
    unsigned long long *slot = reinterpret_cast<unsigned long long *>(sm + b2 + (size_t)bs * nrhs + (3 * bs + nn + 1) / 2 + 1);
    int *bad = reinterpret_cast<int *>(slot + 4);
    for (int i = blockIdx.x; i < nf; i += gridDim.x) {
        const long long k0 = rowpts[i], k1 = rowpts[i + 1];
        for (int k = threadIdx.x; k < nn; k += NT) {
            const int j = f2f[(k + 1) + (size_t)nbf * i];
            int s = -1;
            if (j > 0)
                for (long long q = k0 + 1; q < k1; q++)
                    if (colind[q] == j) { s = (int)q; break; }
            src[k] = s;
        }
        if (threadIdx.x == 0) *bad = 0;
        for (int t = threadIdx.x; t < b2; t += NT) D[t] = Hg[(size_t)b2 * k0 + t];
        for (int t = threadIdx.x; t < bs; t += NT) X[t] = Rg[(size_t)bs * i + t];
        __syncthreads();
        for (int t = threadIdx.x; t < b2 * nn; t += NT) {
            const int k = t / b2, e = t % b2, s = src[k];
            X[bs + (size_t)b2 * k + e] = s >= 0 ? Hg[(size_t)b2 * s + e] : 0.0;
        }
        __syncthreads();
        block_gauss_jordan<NT, true>(D, bs, X, bs, bs, nrhs, pivrow, rowused, slot, bad);
        // unknown r of every right-hand side sits in row pivrow[r]
        for (int t = threadIdx.x; t < bs; t += NT) F[(size_t)bs * i + t] = X[pivrow[t]];
        for (int t = threadIdx.x; t < b2 * nn; t += NT) {
            const int r = t % bs, col = t / bs;
            K[(size_t)b2 * nn * i + t] = X[pivrow[r] + (size_t)bs * (1 + col)];
        }
        if (status && threadIdx.x == 0) status[i] = *bad;
        __syncthreads();
    }
}

// y = x + K gather(x)   (gmres.m:40-44, 69-72); one thread per row of a face
__global__ void dense_matvec_kernel(int nb, int nf, int nbf, const double *__restrict__ K, const int *__restrict__ f2f,
                                    const double *__restrict__ x, double *__restrict__ y) {
    const int nn = nbf - 1;
    const size_t total = (size_t)nb * nf;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(t % nb);
        const size_t i = t / nb;
        double s = x[t];
        for (int k = 0; k < nn; k++) {
            const int j = f2f[(k + 1) + (size_t)nbf * i];
            if (j <= 0) continue;
            const double *Kk = K + (size_t)nb * nb * (k + (size_t)nn * i) + r, *xj = x + (size_t)nb * (j - 1);
            for (int c = 0; c < nb; c++) s += Kk[(size_t)nb * c] * xj[c];
        }
        y[t] = s;
    }
}

// part[v * G + block] = partial sums of V(:, v)' w for v <= j  (classical Gram-Schmidt, gmres.m:80)
__global__ void multi_dot_partial_kernel(size_t n, const double *__restrict__ V, const double *__restrict__ w,
                                         double *__restrict__ part) {
    __shared__ double red[32];
    const int v = blockIdx.y;
    const double *a = V + n * v;
    double s = 0.0;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) s += a[t] * w[t];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) part[(size_t)v * gridDim.x + blockIdx.x] = s;
    }
}

// h[v] = sum of the G partials of vector v (one block per v, fixed order: deterministic)
__global__ void multi_dot_final_kernel(int G, const double *__restrict__ part, double *__restrict__ h) {
    __shared__ double red[32];
    double s = 0.0;
    for (int b = threadIdx.x; b < G; b += blockDim.x) s += part[(size_t)blockIdx.x * G + b];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) h[blockIdx.x] = s;
    }
}

// w -= V(:, 0:nv) h(0:nv)   (gmres.m:81)
__global__ void cgs_update_kernel(size_t n, int nv, const double *__restrict__ V, const double *__restrict__ h,
                                  double *__restrict__ w) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        double s = w[t];
        for (int v = 0; v < nv; v++) s -= V[n * v + t] * h[v];
        w[t] = s;
    }
}

__global__ void copy_scalar_kernel(const double *src, double *dst) { *dst = *src; }

static int n_sm() {
    int d = 0, n = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d);
    return n > 0 ? n : 1;
}

static unsigned grid_n(size_t n, int threads) {
    size_t g = (n + threads - 1) / threads, cap = (size_t)n_sm() * 8;
    if (g > cap) g = cap;
    return (unsigned)(g < 1 ? 1 : g);
}

static int status_of_last_error() {
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : -1000 - (int)e;
}

}  // namespace hdgx

using namespace hdgx;

extern "C" {

int hdgx_arraymul(int rowsA, int colsA, int ndim3, int rowsB, int colsB, int ndimB, const double *A, const double *B,
                  double *C, hdgx_stream_t stream) {
    if (rowsA < 0 || colsA < 0 || ndim3 < 0 || rowsB < 0 || colsB < 0) return -1;
    if (colsA != rowsB) return -1;                       // arraymul.c:45-47
    if ((size_t)rowsA * ndim3 == 0) return 0;
    if (!A || !B || !C) return -1;
    cudaStream_t st = (cudaStream_t)stream;
    if (ndimB == 2 && colsB == ndim3) {
        batched_gemv_kernel<<<grid_n((size_t)rowsA * ndim3, 256), 256, 0, st>>>(rowsA, colsA, ndim3, A, B, C);
    } else {
        if (colsB == 0) return 0;
        batched_gemm_kernel<<<grid_n((size_t)rowsA * colsB * ndim3, 256), 256, 0, st>>>(rowsA, colsA, colsB, ndim3, A, B, C);
    }
    return status_of_last_error();
}

int hdgx_dense_block_system(const hdgx_bsr *A, const double *Hg, const double *Rg, int nbf, const int *f2f, double *K,
                            double *F, int *status, hdgx_stream_t stream) {
    if (!A || !Hg || !Rg || !f2f || !K || !F || nbf < 2 || A->bs < 1 || A->bs > 128) return -1;
    if (A->nf == 0) return 0;
    const int bs = A->bs, nn = nbf - 1, nrhs = 1 + bs * nn;
    const size_t smem = sizeof(double) * ((size_t)bs * bs + (size_t)bs * nrhs + (3 * bs + nn + 1) / 2 + 1 + 4) + sizeof(int) * 2;
    if (smem > 227 * 1024) return -3;
    if (allow_dynamic_smem((const void *)dense_block_kernel<256>, smem) != cudaSuccess) return -10;
    const int grid = A->nf < n_sm() * 4 ? A->nf : n_sm() * 4;
    dense_block_kernel<256><<<grid, 256, smem, (cudaStream_t)stream>>>(bs, A->nf, nbf, A->rowpts, A->colind, Hg, Rg, f2f,
                                                                      K, F, status);
    return status_of_last_error();
}

int hdgx_dense_matvec(int nb, int nf, int nbf, const double *K, const int *f2f, const double *x, double *y,
                      hdgx_stream_t stream) {
    if (nb < 1 || nf < 0 || nbf < 1 || !K || !f2f || !x || !y) return -1;
    if (nf == 0) return 0;
    dense_matvec_kernel<<<grid_n((size_t)nb * nf, 256), 256, 0, (cudaStream_t)stream>>>(nb, nf, nbf, K, f2f, x, y);
    return status_of_last_error();
}

size_t hdgx_gmres_dense_workspace_bytes(int nb, int nf, int restart) {
    if (nb < 1 || nf < 0 || restart < 1) return 0;
    const size_t N = (size_t)nb * nf, m = (size_t)restart;
    return sizeof(double) * (N * (m + 1) + N + (m + 1) * m + 4 * (m + 1) + 8 + 1024 * (m + 1) + (m + 1)) + 256;
}

int hdgx_gmres_dense(int nb, int nf, int nbf, const double *K, const int *f2f, const double *b, double *x, int restart,
                     double tol, int maxit, int *iters, int *flag, double *relres, double *history, void *workspace,
                     hdgx_stream_t stream) {
    if (nb < 1 || nf < 1 || nbf < 1 || !K || !f2f || !b || !x || restart < 1 || maxit < 1) return -1;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t N = (size_t)nb * nf;
    const int m = restart;
    void *mem = workspace;
    bool own = false;
    if (!mem) {
        if (cudaMallocAsync(&mem, hdgx_gmres_dense_workspace_bytes(nb, nf, restart), st) != cudaSuccess) return -13;
        own = true;
    }
    double *V = (double *)mem;
    double *t = V + N * (m + 1);
    GmresState gs;
    gs.H = t + N;
    gs.cs = gs.H + (size_t)(m + 1) * m;
    gs.sn = gs.cs + (m + 1);
    gs.g = gs.sn + (m + 1);
    gs.y = gs.g + (m + 1);
    gs.scal = gs.y + (m + 1);
    gs.hist = nullptr;
    double *part = gs.scal + 8;                  // [1024 * (m + 1)] partial dot products
    const unsigned G = grid_n(N, 256) > 1024 ? 1024 : grid_n(N, 256);
    auto norm_into = [&](const double *v, double *out) {
        dot_partial_kernel<<<G, 256, 0, st>>>(N, v, v, part);
        dot_final_kernel<<<1, 256, 0, st>>>((int)G, part, out, 1);
    };
    double h_s[3] = {0.0, 0.0, 0.0};
    norm_into(b, gs.scal + 2);
    cudaMemcpyAsync(h_s, gs.scal + 2, sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    const double nrmb = h_s[0];
    int iter = 0, fl = 2;
    double res_rel = 0.0;
    if (!(nrmb > 0.0)) fl = 0;
    while (fl == 2) {
        // r = b - A x, beta = |r|, V(:, 0) = r / beta   (gmres.m:38-50)
        dense_matvec_kernel<<<grid_n(N, 256), 256, 0, st>>>(nb, nf, nbf, K, f2f, x, t);
        sub_kernel<<<grid_n(N, 256), 256, 0, st>>>(N, b, t, V);
        norm_into(V, gs.scal + 0);
        cudaMemcpyAsync(h_s, gs.scal + 0, sizeof(double), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        const double beta = h_s[0];
        res_rel = beta / nrmb;
        if (history && iter < maxit) history[iter] = res_rel;
        iter++;
        if (!isfinite(res_rel)) { fl = 3; break; }
        if (res_rel <= tol) { fl = 0; break; }
        if (iter >= maxit) { fl = 1; break; }
        scale_div_kernel<<<grid_n(N, 256), 256, 0, st>>>(N, gs.scal + 0, V, V);
        gmres_init_kernel<<<1, 64, 0, st>>>(gs, m);
        int jdone = 0;
        for (int j = 0; j < m; j++) {
            // the convergence / iteration tests of gmres.m:53-64, made at the top of each inner
            // step (for j = 0 they were made on beta above)
            if (j > 0) {
                if (res_rel <= tol) { fl = 0; break; }
                if (iter >= maxit) { fl = 1; break; }
            }
            double *w = V + N * (j + 1);
            double *hc = gs.H + (size_t)(m + 1) * j;
            dense_matvec_kernel<<<grid_n(N, 256), 256, 0, st>>>(nb, nf, nbf, K, f2f, V + N * j, w);
            // classical Gram-Schmidt: h = V' w, w -= V h   (gmres.m:80-81)
            multi_dot_partial_kernel<<<dim3(G, j + 1), 256, 0, st>>>(N, V, w, part);
            multi_dot_final_kernel<<<j + 1, 256, 0, st>>>((int)G, part, hc);
            cgs_update_kernel<<<grid_n(N, 256), 256, 0, st>>>(N, j + 1, V, hc, w);
            norm_into(w, hc + j + 1);
            copy_scalar_kernel<<<1, 1, 0, st>>>(hc + j + 1, gs.scal + 3);
            scale_div_kernel<<<grid_n(N, 256), 256, 0, st>>>(N, hc + j + 1, w, w);
            givens_kernel<<<1, 1, 0, st>>>(gs, m, j);
            cudaMemcpyAsync(h_s, gs.scal + 1, 3 * sizeof(double), cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
            res_rel = h_s[0] / nrmb;
            if (history && iter < maxit) history[iter] = res_rel;
            iter++;
            jdone = j + 1;
            if (!isfinite(res_rel)) { fl = 3; break; }
            if (!(h_s[2] != 0.0)) break;                 // breakdown: restart from the updated x
        }
        hess_solve_kernel<<<1, 1, 0, st>>>(gs, m, jdone);
        for (int i = 0; i < jdone; i++) axpy_kernel<<<grid_n(N, 256), 256, 0, st>>>(N, gs.y + i, 1.0, V + N * i, x);
    }
    cudaStreamSynchronize(st);
    if (iters) *iters = iter;
    if (flag) *flag = fl;
    if (relres) *relres = res_rel;
    if (own) cudaFreeAsync(mem, st);
    return cudaGetLastError() == cudaSuccess ? 0 : -12;
}

}  // extern "C"
