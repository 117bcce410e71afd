// schur_adjoint.cu -- batched FP64 adjoint (transposed) local Schur complements on the
// reference MEX layouts.
//
// hdgx_schur_uq_adjoint replaces kernel/schur_uq_adjoint.c (mexFunction :300-382,
// localsolveuq :43-298).  With B_n = BD(:,:,:,ncu+(1:ncu)+ncu*n), G_n = GK(:,:,:,ncu+(1:ncu)+ncu*n),
// D = BD(:,:,:,1:ncu), K = GK(:,:,:,1:ncu) as matrices over (r,a) / (a,f) / (s,b) and Mi = inv(M)
// applied to the node index of every component:
//   SDt = D^T + sum_n C_n^T Mi B_n^T          Ru' = Ru + sum_n C_n^T Mi Rq_n
//   [du, dlu] = SDt \ [Ru', -(K^T + sum_n C_n^T Mi G_n^T)]
//   dq_n = Mi (Rq_n - B_n^T du)               dlq_n = -Mi (B_n^T dlu + G_n^T)
//   DUDG = [du, dq]     DUDG_DUH = [dlu, dlq]  (the reference's natural [npv,nc,ncu,ndf] layout)
//   FE = Rh - F^T du - sum_n E_n^T dq_n        AE = H^T + F^T dlu + sum_n E_n^T dlq_n
// (E_n^T dq_n acts on the node index: (E_n^T dq_n)(a,f) = sum_s E(s,f,n) dq_n(s,a)).
// hdgx_schur_u_adjoint replaces kernel/schur_u_adjoint.c (localsolve :43-143, mexFunction :145-212): SDt = D^T,
// [du, dlu] = SDt \ [Ru, -K^T], FE = Rh - F^T du, AE = H^T + F^T dlu; as that MEX writes them,
// du fills the first npv*ncu entries of the element's DUDG slab and dlu (column-major
// [npv*ncu, ncu*ndf]) the first npv*ncu*ncu*ndf entries of its DUDG_DUH slab, the rest zero.
// One CTA per element (grid-stride), runtime sizes, partial pivoting (the reference calls
// dgesv; it factors M with dpotrf, here M is inverted by LU, equal to round-off for the SPD
// mass matrix).  Inputs are never modified (the reference overwrites M, Rq, Ru).
#include <cuda_runtime.h>
#include "hdgx_common.cuh"

namespace hdgx {

struct AdjParams {
    int nd, npv, ncu, nc, ndf, ne, qform, tile;
    const double *M, *C, *E, *BD, *F, *GK, *H, *Rq, *Ru, *Rh;
    double *DUDG, *DUDG_DUH, *AE, *FE;
    int *status;
};

struct AdjPlan {
    size_t M, Mi, W, SD, R, dq, T, ints, bytes;
    __host__ __device__ static AdjPlan make(int nd, int npv, int ncu, int ndf, int qform, int tile) {
        AdjPlan p;
        const size_t nu = (size_t)npv * ncu, nh = (size_t)ncu * ndf, q = qform ? 1 : 0;
        p.M = 0;
        p.Mi = p.M + q * npv * npv;
        p.W = p.Mi + q * npv * npv;                       // W_n = C_n^T Mi  [npv, npv, nd]
        p.SD = p.W + q * npv * npv * nd;
        p.R = p.SD + nu * nu;
        p.dq = p.R + nu * (1 + nh);                       // t_n, then dq_n  [nu, nd]
        p.T = p.dq + q * nu * nd;                         // dlq tile [nu, nd, tile] (+ pre-image)
        const size_t nd_ = p.T + q * 2 * nu * nd * (size_t)tile;
        p.ints = nd_;
        p.bytes = sizeof(double) * nd_ + sizeof(int) * (nu + npv + 1);
        return p;
    }
};

template <int NT>
__global__ void __launch_bounds__(NT) schur_adjoint_kernel(const __grid_constant__ AdjParams P) {
    extern __shared__ __align__(16) double sm[];
    const int nd = P.nd, npv = P.npv, ncu = P.ncu, nc = P.nc, ndf = P.ndf, tid = threadIdx.x;
    const int nu = npv * ncu, nh = ncu * ndf, nq = npv * nc;
    const AdjPlan L = AdjPlan::make(nd, npv, ncu, ndf, P.qform, P.tile);
    double *sM = sm + L.M, *sMi = sm + L.Mi, *sW = sm + L.W, *sSD = sm + L.SD, *sR = sm + L.R;
    double *sdq = sm + L.dq, *sT = sm + L.T;
    int *ipiv = reinterpret_cast<int *>(sm + L.ints), *ipivM = ipiv + nu, *sbad = ipivM + npv;

    for (int e = blockIdx.x; e < P.ne; e += gridDim.x) {
        const double *BD = P.BD + (size_t)e * nu * npv * nc;   // [npv, ncu, npv, nc]
        const double *GK = P.GK + (size_t)e * nh * npv * nc;   // [ncu, ndf, npv, nc]
        const double *F = P.F + (size_t)e * nu * nh;           // [npv, ncu, ncu, ndf]
        const double *H = P.H + (size_t)e * nh * nh;
        const double *Rq = P.qform ? P.Rq + (size_t)e * nu * nd : nullptr;   // [npv, ncu, nd]
        // B_n((r,a),(s,b)) and G_n((a,f),(s,b)) in global memory
        auto Bn = [&](int r, int a, int s, int b, int n) {
            return BD[r + npv * a + (size_t)nu * s + (size_t)nu * npv * (ncu + b + ncu * n)];
        };
        auto Gn = [&](int af, int s, int b, int n) {
            return GK[af + (size_t)nh * s + (size_t)nh * npv * (ncu + b + ncu * n)];
        };
        if (tid == 0) *sbad = 0;
        if (P.qform) {
            for (int i = tid; i < npv * npv; i += NT) {
                sM[i] = P.M[(size_t)e * npv * npv + i];
                sMi[i] = (i % npv == i / npv) ? 1.0 : 0.0;
            }
            __syncthreads();
            block_lu<NT>(sM, npv, npv, ipivM, sbad);
            if (tid == 0 && *sbad) *sbad = 1;
            __syncthreads();
            block_lu_solve<NT>(sM, npv, npv, ipivM, sMi, npv, npv);
            __syncthreads();
            const double *C = P.C + (size_t)e * npv * npv * nd;
            for (int i = tid; i < npv * npv * nd; i += NT) {      // W_n(s, t) = sum_u C_n(u, s) Mi(u, t)
                const int s = i % npv, t = (i / npv) % npv, n = i / (npv * npv);
                double v = 0.0;
                for (int u = 0; u < npv; u++) v += C[u + npv * (s + npv * n)] * sMi[u + npv * t];
                sW[i] = v;
            }
            __syncthreads();
        }
        // SDt((s,b),(r,a)) = D((r,a),(s,b)) + sum_n sum_t W_n(s,t) B_n((r,a),(t,b))
        for (int i = tid; i < nu * nu; i += NT) {
            const int s = i % npv, b = (i / npv) % ncu, ra = i / nu, r = ra % npv, a = ra / npv;
            double v = BD[r + npv * a + (size_t)nu * s + (size_t)nu * npv * b];
            if (P.qform)
                for (int n = 0; n < nd; n++)
                    for (int t = 0; t < npv; t++) v += sW[s + npv * (t + npv * n)] * Bn(r, a, t, b, n);
            sSD[i] = v;
        }
        // R(:,0) = Ru + sum_n W_n Rq_n;  R(:,1+(a,f)) = -(K^T + sum_n W_n G_n^T)
        for (int i = tid; i < nu; i += NT) {
            const int s = i % npv, b = i / npv;
            double v = P.Ru[(size_t)e * nu + i];
            if (P.qform)
                for (int n = 0; n < nd; n++)
                    for (int t = 0; t < npv; t++) v += sW[s + npv * (t + npv * n)] * Rq[t + npv * (b + ncu * n)];
            sR[i] = v;
        }
        for (int i = tid; i < nu * nh; i += NT) {
            const int s = i % npv, b = (i / npv) % ncu, af = i / nu;
            double v = GK[af + (size_t)nh * s + (size_t)nh * npv * b];
            if (P.qform)
                for (int n = 0; n < nd; n++)
                    for (int t = 0; t < npv; t++) v += sW[s + npv * (t + npv * n)] * Gn(af, t, b, n);
            sR[nu + i] = -v;
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
        const double *du = sR, *dlu = sR + nu;
        double *gd = P.DUDG + (size_t)e * nq;
        double *gdd = P.DUDG_DUH + (size_t)e * nq * nh;
        double *gae = P.AE + (size_t)e * nh * nh;
        if (P.qform) {
            // dq_n = Mi (Rq_n - B_n^T du)
            for (int i = tid; i < nu * nd; i += NT) {
                const int s = i % npv, b = (i / npv) % ncu, n = i / nu;
                double v = Rq[s + npv * (b + ncu * n)];
                for (int ra = 0; ra < nu; ra++) v -= Bn(ra % npv, ra / npv, s, b, n) * du[ra];
                sT[i] = v;
            }
            __syncthreads();
            for (int i = tid; i < nu * nd; i += NT) {
                const int s = i % npv, bn = i / npv;
                double v = 0.0;
                for (int t = 0; t < npv; t++) v += sMi[s + npv * t] * sT[t + npv * bn];
                sdq[i] = v;
            }
            __syncthreads();
            for (int i = tid; i < nq; i += NT) gd[i] = i < nu ? du[i] : sdq[i - nu];
        } else {
            for (int i = tid; i < nq; i += NT) gd[i] = i < nu ? du[i] : 0.0;
        }
        // FE = Rh - F^T du (- sum_n E_n^T dq_n)
        for (int i = tid; i < nh; i += NT) {
            const int a = i % ncu, f = i / ncu;
            double v = P.Rh[(size_t)e * nh + i];
            for (int rb = 0; rb < nu; rb++) v -= F[rb + (size_t)nu * i] * du[rb];
            if (P.qform) {
                const double *E = P.E + (size_t)e * npv * ndf * nd;
                double t = 0.0;
                for (int n = 0; n < nd; n++)
                    for (int s = 0; s < npv; s++) t += E[s + npv * (f + ndf * n)] * sdq[s + npv * (a + ncu * n)];
                v -= t;
            }
            P.FE[(size_t)e * nh + i] = v;
        }
        if (!P.qform) {
            // the u form's packed outputs: dlu column-major into the slab's first nu*nh entries
            for (size_t i = tid; i < (size_t)nq * nh; i += NT) gdd[i] = i < (size_t)nu * nh ? dlu[i] : 0.0;
            for (int i = tid; i < nh * nh; i += NT) {
                const int af = i % nh, k = i / nh;
                double v = H[k + (size_t)nh * af];
                for (int rb = 0; rb < nu; rb++) v += F[rb + (size_t)nu * af] * dlu[rb + (size_t)nu * k];
                gae[i] = v;
            }
        } else {
            const double *E = P.E + (size_t)e * npv * ndf * nd;
            double *sY = sT + (size_t)nu * nd * P.tile;
            for (int k0 = 0; k0 < nh; k0 += P.tile) {
                const int nt = min(P.tile, nh - k0);
                // y_n = B_n^T dlu_k + G_n^T_k, then dlq_n = -Mi y_n, for the tile's columns k
                for (int i = tid; i < nu * nd * nt; i += NT) {
                    const int s = i % npv, b = (i / npv) % ncu, n = (i / nu) % nd, t = i / (nu * nd), k = k0 + t;
                    double v = Gn(k, s, b, n);
                    for (int ra = 0; ra < nu; ra++) v += Bn(ra % npv, ra / npv, s, b, n) * dlu[ra + (size_t)nu * k];
                    sY[i] = v;
                }
                __syncthreads();
                for (int i = tid; i < nu * nd * nt; i += NT) {
                    const int s = i % npv, rest = i / npv;
                    double v = 0.0;
                    for (int u = 0; u < npv; u++) v -= sMi[s + npv * u] * sY[u + npv * rest];
                    sT[i] = v;
                }
                __syncthreads();
                for (int i = tid; i < nq * nt; i += NT) {          // DUDG_DUH(:, :, k)
                    const int rc = i % nq, t = i / nq, k = k0 + t;
                    gdd[(size_t)nq * k + rc] = rc < nu ? dlu[rc + (size_t)nu * k] : sT[(rc - nu) + (size_t)nu * nd * t];
                }
                for (int i = tid; i < nh * nt; i += NT) {          // AE(:, k)
                    const int af = i % nh, t = i / nh, k = k0 + t, a = af % ncu, f = af / ncu;
                    double v = H[k + (size_t)nh * af];
                    for (int rb = 0; rb < nu; rb++) v += F[rb + (size_t)nu * af] * dlu[rb + (size_t)nu * k];
                    double w = 0.0;
                    for (int n = 0; n < nd; n++)
                        for (int s = 0; s < npv; s++)
                            w += E[s + npv * (f + ndf * n)] * sT[s + npv * (a + ncu * n) + (size_t)nu * nd * t];
                    gae[(size_t)nh * k + af] = v + w;
                }
                __syncthreads();
            }
        }
        if (tid == 0 && P.status) P.status[e] = *sbad;
        __syncthreads();
    }
}

int schur_adjoint_launch(int qform, int nd, int npv, int ncu, int nc, int ndf, int ne, const double *M,
                         const double *C, const double *E, const double *BD, const double *F, const double *GK,
                         const double *H, const double *Rq, const double *Ru, const double *Rh, double *DUDG,
                         double *DUDG_DUH, double *AE, double *FE, int *status, cudaStream_t st) {
    constexpr int NT = 256;
    AdjParams p{nd, npv, ncu, nc, ndf, ne, qform, 1, M, C, E, BD, F, GK, H, Rq, Ru, Rh, DUDG, DUDG_DUH, AE, FE, status};
    int tile = ncu * ndf;
    AdjPlan L = AdjPlan::make(nd, npv, ncu, ndf, qform, tile);
    while (L.bytes > 200 * 1024 && tile > 1) {
        tile = (tile + 1) / 2;
        L = AdjPlan::make(nd, npv, ncu, ndf, qform, tile);
    }
    if (L.bytes > 227 * 1024) return -3;
    p.tile = tile;
    auto kern = schur_adjoint_kernel<NT>;
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
