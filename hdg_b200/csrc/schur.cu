// schur.cu -- batched FP64 local Schur complements on the reference MEX layouts.
//
// hdgx_schur_uq replaces kernel/schur_uq.c (mexFunction :193-287, localsolveuq :42-191;
// MATLAB twin kernel/schur_primal.m:52-150): per element
//   Mi = inv(M); SD = D + B Mi C; du = SD \ (Ru - B Mi Rq); dlu = SD \ (B Mi E - F)
//   DUDG = [du, Mi Rq + Mi C du]; DUDG_DUH = [dlu, Mi C dlu - Mi E (x) I]
//   FE = Rh - GK DUDG; AE = H + GK DUDG_DUH.
// hdgx_schur_u replaces kernel/schur_u.c (:42-163; MATLAB twin schur_primal.m:13-49).
// One CTA per element (grid-stride), runtime sizes, operands staged in shared memory; the
// inputs are never modified (the reference MEX overwrites M, C, E, BD, F, Rq, Ru).
#include <cuda_runtime.h>
#include "hdgx_common.cuh"

namespace hdgx {

struct SchurParams {
    int nd, npv, ncu, nc, ndf, ne, qform;   // qform 1: (u,q) form, 0: u only
    const double *M, *C, *E, *BD, *F, *GK, *H, *Rq, *Ru, *Rh;
    double *DUDG, *DUDG_DUH, *AE, *FE;
    int *status;
    int tile;
};

struct SchurPlan {
    size_t M, Mi, SD, R, dudg, X, ints, bytes;
    __host__ __device__ static SchurPlan make(int nd, int npv, int ncu, int nc, int ndf, int tile) {
        SchurPlan p;
        const size_t nu = (size_t)npv * ncu, nh = (size_t)ncu * ndf, nq = (size_t)npv * nc;
        p.M = 0;
        p.Mi = p.M + (size_t)npv * npv;
        p.SD = p.Mi + (size_t)npv * (npv * nd + ndf * nd + ncu * nd);
        p.R = p.SD + nu * nu;
        p.dudg = p.R + nu * (1 + nh);
        p.X = p.dudg + nq;
        size_t nd_ = p.X + nq * (size_t)tile;
        p.ints = nd_;
        p.bytes = sizeof(double) * nd_ + sizeof(int) * (nu + npv + 1);
        return p;
    }
};

template <int NT>
__global__ void __launch_bounds__(NT) schur_kernel(const __grid_constant__ SchurParams P) {
    extern __shared__ __align__(16) double sm[];
    const int nd = P.nd, npv = P.npv, ncu = P.ncu, nc = P.nc, ndf = P.ndf;
    const int nu = npv * ncu, nh = ncu * ndf, nq = npv * nc, tid = threadIdx.x;
    const SchurPlan L = SchurPlan::make(nd, npv, ncu, nc, ndf, P.tile);
    double *sM = sm + L.M, *sMi = sm + L.Mi, *sSD = sm + L.SD, *sR = sm + L.R;
    double *sdudg = sm + L.dudg, *sX = sm + L.X;
    int *ipiv = reinterpret_cast<int *>(sm + L.ints), *ipivM = ipiv + nu, *sbad = ipivM + npv;
    const int ncolMi = npv * nd + ndf * nd + ncu * nd;
    double *sMiC = sMi, *sMiE = sMi + npv * npv * nd, *sMiRq = sMiE + npv * ndf * nd;

    for (int e = blockIdx.x; e < P.ne; e += gridDim.x) {
        const double *BD = P.BD + (size_t)e * nu * nq;
        const double *F = P.F + (size_t)e * nu * nh;
        const double *GK = P.GK + (size_t)e * nh * nq;
        const double *H = P.H + (size_t)e * nh * nh;
        if (tid == 0) *sbad = 0;
        // D -> SD; Ru -> R(:,0); -F -> R(:,1:)
        for (int i = tid; i < nu * nu; i += NT) sSD[i] = BD[i];
        for (int i = tid; i < nu; i += NT) sR[i] = P.Ru[(size_t)e * nu + i];
        for (int i = tid; i < nu * nh; i += NT) sR[nu + i] = -F[i];
        if (P.qform) {
            for (int i = tid; i < npv * npv; i += NT) sM[i] = P.M[(size_t)e * npv * npv + i];
            for (int i = tid; i < npv * npv * nd; i += NT) sMiC[i] = P.C[(size_t)e * npv * npv * nd + i];
            for (int i = tid; i < npv * ndf * nd; i += NT) sMiE[i] = P.E[(size_t)e * npv * ndf * nd + i];
            for (int i = tid; i < npv * ncu * nd; i += NT) sMiRq[i] = P.Rq[(size_t)e * npv * ncu * nd + i];
            __syncthreads();
            block_lu<NT>(sM, npv, npv, ipivM, sbad);
            if (tid == 0 && *sbad) *sbad = 1;
            __syncthreads();
            block_lu_solve<NT>(sM, npv, npv, ipivM, sMi, npv, ncolMi);
            __syncthreads();
            // B(ia, j, b, d) = BD(ia, j, ncu + b + ncu*d) read from global
            const double *B = BD + (size_t)nu * nu;
            for (int i = tid; i < nu * nu; i += NT) {           // SD += B Mi C
                const int ia = i % nu, k = (i / nu) % npv, b = i / (nu * npv);
                double v = 0.0;
                for (int d = 0; d < nd; d++)
                    for (int j = 0; j < npv; j++)
                        v += B[ia + (size_t)nu * (j + npv * (b + ncu * d))] * sMiC[j + npv * (k + npv * d)];
                sSD[i] += v;
            }
            for (int ia = tid; ia < nu; ia += NT) {             // R0 -= B Mi Rq
                double v = 0.0;
                for (int k = 0; k < nu * nd; k++) v += B[ia + (size_t)nu * k] * sMiRq[k];
                sR[ia] -= v;
            }
            for (int i = tid; i < nu * nh; i += NT) {           // R += B Mi E
                const int ia = i % nu, b = (i / nu) % ncu, f = i / (nu * ncu);
                double v = 0.0;
                for (int d = 0; d < nd; d++)
                    for (int j = 0; j < npv; j++)
                        v += B[ia + (size_t)nu * (j + npv * (b + ncu * d))] * sMiE[j + npv * (f + ndf * d)];
                sR[nu + i] += v;
            }
        }
        __syncthreads();
        {
            const int before = *sbad;
            __syncthreads();
            block_lu<NT>(sSD, nu, nu, ipiv, sbad);
            if (tid == 0 && *sbad && !before) *sbad = 2;
            __syncthreads();
            block_lu_solve<NT>(sSD, nu, nu, ipiv, sR, nu, 1 + nh);
            __syncthreads();
        }
        // DUDG
        double *gd = P.DUDG + (size_t)e * nq;
        for (int i = tid; i < nq; i += NT) {
            const int r = i % npv, c = i / npv;
            double v = 0.0;
            if (c < ncu) v = sR[r + npv * c];
            else if (P.qform) {
                const int a = (c - ncu) % ncu, d = (c - ncu) / ncu;
                v = sMiRq[r + npv * (a + ncu * d)];
                for (int s = 0; s < npv; s++) v += sMiC[r + npv * (s + npv * d)] * sR[s + npv * a];
            }
            sdudg[i] = v;
            gd[i] = v;
        }
        __syncthreads();
        for (int i = tid; i < nh; i += NT) {                     // FE = Rh - GK DUDG
            double v = 0.0;
            for (int k = 0; k < nq; k++) v += GK[i + (size_t)nh * k] * sdudg[k];
            P.FE[(size_t)e * nh + i] = P.Rh[(size_t)e * nh + i] - v;
        }
        // DUDG_DUH and AE in column tiles
        double *gdd = P.DUDG_DUH + (size_t)e * nq * nh;
        double *gae = P.AE + (size_t)e * nh * nh;
        for (int k0 = 0; k0 < nh; k0 += P.tile) {
            const int nt = min(P.tile, nh - k0);
            for (int i = tid; i < nq * nt; i += NT) {
                const int rc = i % nq, t = i / nq, k = k0 + t, r = rc % npv, c = rc / npv;
                const double *dlu = sR + (size_t)nu * (1 + k);
                double v = 0.0;
                if (c < ncu) v = dlu[r + npv * c];
                else if (P.qform) {
                    const int a = (c - ncu) % ncu, d = (c - ncu) / ncu, b = k % ncu, f = k / ncu;
                    v = (a == b) ? -sMiE[r + npv * (f + ndf * d)] : 0.0;
                    for (int s = 0; s < npv; s++) v += sMiC[r + npv * (s + npv * d)] * dlu[s + npv * a];
                }
                sX[i] = v;
                gdd[(size_t)nq * k0 + i] = v;
            }
            __syncthreads();
            for (int i = tid; i < nh * nt; i += NT) {
                const int row = i % nh, t = i / nh, k = k0 + t;
                double v = H[row + (size_t)nh * k];
                for (int q = 0; q < nq; q++) v += GK[row + (size_t)nh * q] * sX[q + nq * t];
                gae[(size_t)nh * k0 + i] = v;
            }
            __syncthreads();
        }
        if (tid == 0 && P.status) P.status[e] = *sbad;
        __syncthreads();
    }
}

int schur_launch(int qform, int nd, int npv, int ncu, int nc, int ndf, int ne, const double *M,
                 const double *C, const double *E, const double *BD, const double *F, const double *GK,
                 const double *H, const double *Rq, const double *Ru, const double *Rh, double *DUDG,
                 double *DUDG_DUH, double *AE, double *FE, int *status, cudaStream_t st) {
    constexpr int NT = 256;
    SchurParams p{nd, npv, ncu, nc, ndf, ne, qform, M, C, E, BD, F, GK, H, Rq, Ru, Rh,
                  DUDG, DUDG_DUH, AE, FE, status, 1};
    int tile = ncu * ndf;
    SchurPlan L = SchurPlan::make(nd, npv, ncu, nc, ndf, tile);
    while (L.bytes > 200 * 1024 && tile > 1) {
        tile = (tile + 1) / 2;
        L = SchurPlan::make(nd, npv, ncu, nc, ndf, tile);
    }
    if (L.bytes > 227 * 1024) return -3;
    p.tile = tile;
    auto kern = schur_kernel<NT>;
    if (allow_dynamic_smem((const void *)kern, L.bytes) != cudaSuccess) return -10;
    int dev = 0, nsm = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, L.bytes);
    if (per_sm < 1) return -11;
    int grid = nsm * per_sm;
    if (grid > ne) grid = ne;
    if (grid < 1) return 0;
    kern<<<grid, NT, L.bytes, st>>>(p);
    return cudaGetLastError() == cudaSuccess ? 0 : -12;
}

}  // namespace hdgx
