/*
 * oracle_global.c -- CPU restatement of the reference's condensed (trace) system path.
 * TEST INFRASTRUCTURE ONLY (the parity oracle and CPU baseline; never called by the
 * product library).
 *
 *   orc_globalassembly  kernel/globalassembly.m:21-37  block-CSR Hg[bs,bs,nnzb], Rg[bs,nf]
 *                       by face rows (bs = ncu*npf).  Trace dofs are placed where the active
 *                       sparse assembly kernel/hdg_assemble.m:77-87 puts them (global dof
 *                       elcon(n,a,e)); see the note at the function.
 *   orc_matvec          kernel/matvec.m:8-12
 *   orc_mdf_ordering    kernel/computeMDFordering.m:13-161
 *   orc_bilu0           kernel/computeBILU0.m:11-46   (ordered block ILU(0), right-looking,
 *                       diagonal blocks stored inverted)
 *   orc_bilu0_apply     kernel/applyBILU0.m:10-48
 *   orc_gmres_bilu0     kernel/gmres_bilu0.m:17-105  (left preconditioned, restarted,
 *                       modified Gram-Schmidt; the Hessenberg least-squares problem
 *                       y = H \ (beta e1) is solved with Givens rotations, which gives the
 *                       same minimiser and residual)
 *   orc_dense_block_system  mesh/mkmesh/mkf2f.m + kernel/mkDenseBlockSystem.m:9-95
 *   orc_dense_matvec        kernel/gmres.m:40-44
 *   orc_gmres_dense         kernel/gmres.m:1-111 (classical Gram-Schmidt)
 * Index conventions: rowpts 0-based offsets [nf+1], colind 1-based [nnzb], diagonal first;
 * elcon [npf*nfe, ne] 1-based; t2f [ne, nfe] 1-based (column-major); orderings 0-based.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* small dense helpers (column-major, n x n) */
static void mm(int n, const double *A, const double *B, double *C)       /* C = A B */
{
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
            double s = 0.0;
            for (int k = 0; k < n; k++) s += A[i + n * k] * B[k + n * j];
            C[i + n * j] = s;
        }
}

static void mm_sub(int n, const double *A, const double *B, double *C)   /* C -= A B */
{
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
            double s = 0.0;
            for (int k = 0; k < n; k++) s += A[i + n * k] * B[k + n * j];
            C[i + n * j] -= s;
        }
}

static int inv_inplace(int n, double *A)                                   /* A = inv(A), LU with pivoting */
{
    double *W = malloc(sizeof(double) * n * n);
    int *piv = malloc(sizeof(int) * n), rc = 0;
    memcpy(W, A, sizeof(double) * n * n);
    for (int k = 0; k < n; k++) {
        int p = k; double mx = fabs(W[k + n * k]);
        for (int i = k + 1; i < n; i++) if (fabs(W[i + n * k]) > mx) { mx = fabs(W[i + n * k]); p = i; }
        piv[k] = p;
        if (mx == 0.0 || !isfinite(mx)) { rc = k + 1; break; }
        if (p != k) for (int j = 0; j < n; j++) { double t = W[k + n * j]; W[k + n * j] = W[p + n * j]; W[p + n * j] = t; }
        for (int i = k + 1; i < n; i++) W[i + n * k] /= W[k + n * k];
        for (int j = k + 1; j < n; j++) for (int i = k + 1; i < n; i++) W[i + n * j] -= W[i + n * k] * W[k + n * j];
    }
    if (!rc) {
        for (int c = 0; c < n; c++) {
            double *b = A + n * c;
            for (int i = 0; i < n; i++) b[i] = (i == c) ? 1.0 : 0.0;
            for (int k = 0; k < n; k++) if (piv[k] != k) { double t = b[k]; b[k] = b[piv[k]]; b[piv[k]] = t; }
            for (int k = 0; k < n; k++) for (int i = k + 1; i < n; i++) b[i] -= W[i + n * k] * b[k];
            for (int k = n - 1; k >= 0; k--) { b[k] /= W[k + n * k]; for (int i = 0; i < k; i++) b[i] -= W[i + n * k] * b[k]; }
        }
    }
    free(W); free(piv);
    return rc;
}

/* globalassembly.m:21-37.  The reference reads the element block with the face-local
 * positions ind = elcon(:,a,e) - (i-1)*npf used as a gather index; in 2D the position map
 * between two neighbours is the identity or a reversal (its own inverse), so that equals
 * placing element node n at face position ind(n), which is what the active sparse assembly
 * (hdg_assemble.m:77-87, dof elcon(n,a,e)) does in every dimension.  This routine places
 * by elcon, i.e. Hg(:, ind(n), :, ind(n'), k) += AE(:, n, :, n') for the face pair. */
void orc_globalassembly(int ne, int nfe, int npf, int ncu, const int *t2f, const int *elcon,
                        int nf, const long long *rowpts, const int *colind,
                        const double *AE, const double *FE, double *Hg, double *Rg)
{
    const int bs = ncu * npf, ndf = npf * nfe, nh = ncu * ndf;
    const long long nnzb = rowpts[nf];
    memset(Hg, 0, sizeof(double) * bs * bs * (size_t)nnzb);
    memset(Rg, 0, sizeof(double) * bs * (size_t)nf);
    for (int e = 0; e < ne; e++) {
        const double *ae = AE + (size_t)nh * nh * e, *fe = FE + (size_t)nh * e;
        for (int a = 0; a < nfe; a++) {
            const int i = t2f[e + ne * a] - 1;
            for (int n = 0; n < npf; n++) {
                const int mi = elcon[(n + npf * a) + ndf * e] - 1 - npf * i;
                for (int c = 0; c < ncu; c++) Rg[(c + ncu * mi) + bs * (size_t)i] += fe[c + ncu * (n + npf * a)];
            }
            for (int b = 0; b < nfe; b++) {
                const int j = t2f[e + ne * b] - 1;
                long long k = rowpts[i];
                for (; k < rowpts[i + 1]; k++) if (colind[k] - 1 == j) break;
                double *H = Hg + (size_t)bs * bs * k;
                for (int np = 0; np < npf; np++) {
                    const int mj = elcon[(np + npf * b) + ndf * e] - 1 - npf * j;
                    for (int cp = 0; cp < ncu; cp++)
                        for (int n = 0; n < npf; n++) {
                            const int mi = elcon[(n + npf * a) + ndf * e] - 1 - npf * i;
                            for (int c = 0; c < ncu; c++)
                                H[(c + ncu * mi) + bs * (cp + ncu * mj)] +=
                                    ae[(c + ncu * (n + npf * a)) + nh * (cp + ncu * (np + npf * b))];
                        }
                }
            }
        }
    }
}

/* matvec.m: y = Hg x for block-CSR Hg; x, y [bs, nf]. */
void orc_matvec(int nf, int bs, const long long *rowpts, const int *colind, const double *Hg,
                const double *x, double *y)
{
    for (int i = 0; i < nf; i++) {
        double *yi = y + (size_t)bs * i;
        for (int r = 0; r < bs; r++) yi[r] = 0.0;
        for (long long k = rowpts[i]; k < rowpts[i + 1]; k++) {
            const double *H = Hg + (size_t)bs * bs * k, *xj = x + (size_t)bs * (colind[k] - 1);
            for (int c = 0; c < bs; c++) { double xc = xj[c]; for (int r = 0; r < bs; r++) yi[r] += H[r + bs * c] * xc; }
        }
    }
}

static long long find_col(const long long *rowpts, const int *colind, int row, int col1)
{
    for (long long k = rowpts[row]; k < rowpts[row + 1]; k++) if (colind[k] == col1) return k;
    return -1;
}

/* computeBILU0.m:11-46 with a given ordering (o2u[j] = row pivoted at step j, u2o inverse,
 * 0-based).  Mg = Hg on entry (same storage allowed); returns 0 or 1 + step of a singular
 * diagonal block. */
int orc_bilu0(int nf, int bs, const long long *rowpts, const int *colind, const int *o2u,
              const int *u2o, double *Mg)
{
    double *T = malloc(sizeof(double) * bs * bs);
    const size_t b2 = (size_t)bs * bs;
    int rc = 0;
    for (int j = 0; j < nf; j++) {
        const int rj = o2u[j];
        const long long jj = rowpts[rj];
        if (inv_inplace(bs, Mg + b2 * jj) && !rc) rc = j + 1;
        for (long long i = rowpts[rj] + 1; i < rowpts[rj + 1]; i++) {
            const int ri = colind[i] - 1;
            if (u2o[ri] <= j) continue;
            const long long ij = find_col(rowpts, colind, ri, rj + 1);
            mm(bs, Mg + b2 * ij, Mg + b2 * jj, T);                 /* Lij = Hij inv(Ujj) */
            memcpy(Mg + b2 * ij, T, sizeof(double) * b2);
            const long long ii = rowpts[ri];
            mm_sub(bs, Mg + b2 * ij, Mg + b2 * i, Mg + b2 * ii);   /* Uii -= Lij Uji */
            for (long long l = rowpts[ri] + 1; l < rowpts[ri + 1]; l++) {
                const int rij = colind[l] - 1;
                if (u2o[rij] <= j) continue;
                for (long long m = rowpts[rj] + 1; m < rowpts[rj + 1]; m++)
                    if (colind[m] - 1 == rij) mm_sub(bs, Mg + b2 * ij, Mg + b2 * m, Mg + b2 * l);
            }
        }
    }
    free(T);
    return rc;
}

/* applyBILU0.m:10-48: v = (LU)^{-1} x. */
void orc_bilu0_apply(int nf, int bs, const long long *rowpts, const int *colind, const int *o2u,
                     const int *u2o, const double *Mg, const double *x, double *v)
{
    const size_t b2 = (size_t)bs * bs;
    double *y = malloc(sizeof(double) * bs * (size_t)nf), *t = malloc(sizeof(double) * bs);
    for (int j = 0; j < nf; j++) {
        const int rj = o2u[j];
        double *yj = y + (size_t)bs * rj;
        for (int r = 0; r < bs; r++) yj[r] = x[(size_t)bs * rj + r];
        for (long long k = rowpts[rj] + 1; k < rowpts[rj + 1]; k++) {
            const int ri = colind[k] - 1;
            if (u2o[ri] < j) {
                const double *L = Mg + b2 * k, *yi = y + (size_t)bs * ri;
                for (int c = 0; c < bs; c++) for (int r = 0; r < bs; r++) yj[r] -= L[r + bs * c] * yi[c];
            }
        }
    }
    for (int jr = nf - 1; jr >= 0; jr--) {
        const int rj = o2u[jr];
        for (int r = 0; r < bs; r++) t[r] = y[(size_t)bs * rj + r];
        for (long long k = rowpts[rj] + 1; k < rowpts[rj + 1]; k++) {
            const int ri = colind[k] - 1;
            if (u2o[ri] > u2o[rj]) {
                const double *U = Mg + b2 * k, *vi = v + (size_t)bs * ri;
                for (int c = 0; c < bs; c++) for (int r = 0; r < bs; r++) t[r] -= U[r + bs * c] * vi[c];
            }
        }
        const double *Di = Mg + b2 * rowpts[rj];
        double *vj = v + (size_t)bs * rj;
        for (int r = 0; r < bs; r++) { double s = 0.0; for (int c = 0; c < bs; c++) s += Di[r + bs * c] * t[c]; vj[r] = s; }
    }
    free(y); free(t);
}

/* computeMDFordering.m: minimum discarded fill ordering; o2u/u2o 0-based outputs. */
void orc_mdf_ordering(int nf, int bs, const long long *rowpts, const int *colind, const double *Hg,
                      int *o2u, int *u2o)
{
    const size_t b2 = (size_t)bs * bs;
    const long long nnzb = rowpts[nf];
    double *C = calloc(nnzb, sizeof(double)), *w = calloc(nf, sizeof(double));
    double *Di = malloc(sizeof(double) * b2), *T = malloc(sizeof(double) * b2);
    for (int i = 0; i < nf; i++) {
        memcpy(Di, Hg + b2 * rowpts[i], sizeof(double) * b2);
        inv_inplace(bs, Di);
        for (long long n = rowpts[i]; n < rowpts[i + 1]; n++) {
            mm(bs, Di, Hg + b2 * n, T);
            double s = 0.0;
            for (size_t q = 0; q < b2; q++) s += T[q] * T[q];
            C[n] = sqrt(s);
        }
    }
    const double big = 1e100;
    /* weight of row k over the neighbours that are still unnumbered (all, initially) */
    #define ROW_WEIGHT(k, OUT) do {                                                           \
        double acc = 0.0;                                                                     \
        for (long long ni = rowpts[k] + 1; ni < rowpts[k + 1]; ni++) {                          \
            const int ri = colind[ni] - 1;                                                    \
            if (w[ri] >= big) continue;                                                       \
            const long long ik = find_col(rowpts, colind, ri, (k) + 1);                       \
            for (long long nj = rowpts[k] + 1; nj < rowpts[k + 1]; nj++) {                      \
                const int rj = colind[nj] - 1;                                                \
                if (nj == ni || w[rj] >= big) continue;                                       \
                if (find_col(rowpts, colind, ri, rj + 1) < 0) { double d = C[ik] * C[nj]; acc += d * d; } \
            }                                                                                 \
        }                                                                                     \
        OUT = sqrt(acc);                                                                      \
    } while (0)
    for (int k = 0; k < nf; k++) { double v; ROW_WEIGHT(k, v); w[k] = v; }
    for (int l = 0; l < nf; l++) {
        int p = 0; double mn = w[0];
        for (int k = 1; k < nf; k++) if (w[k] < mn) { mn = w[k]; p = k; }
        o2u[l] = p;
        w[p] = big;
        for (long long e = rowpts[p] + 1; e < rowpts[p + 1]; e++) {
            const int k = colind[e] - 1;
            if (w[k] < big) { double v; ROW_WEIGHT(k, v); w[k] = v; }
        }
    }
    #undef ROW_WEIGHT
    for (int i = 0; i < nf; i++) u2o[o2u[i]] = i;
    free(C); free(w); free(Di); free(T);
}

static double nrm2(size_t n, const double *x) { double s = 0.0; for (size_t i = 0; i < n; i++) s += x[i] * x[i]; return sqrt(s); }

/* gmres_bilu0.m: x (in/out, [bs,nf]); returns iterations, *flag 0 converged / 1 maxit,
 * rev[maxit] relative residual history (may be NULL). */
int orc_gmres_bilu0(int nf, int bs, const long long *rowpts, const int *colind, const int *o2u,
                    const int *u2o, const double *Mg, const double *Hg, const double *b, double *x,
                    int restart, double tol, int maxit, int *flag, double *rev)
{
    const size_t N = (size_t)bs * nf;
    double *pb = malloc(sizeof(double) * N), *r = malloc(sizeof(double) * N), *t = malloc(sizeof(double) * N);
    double *V = malloc(sizeof(double) * N * (restart + 1));
    double *Hh = calloc((size_t)(restart + 1) * restart, sizeof(double));
    double *cs = calloc(restart, sizeof(double)), *sn = calloc(restart, sizeof(double)), *g = calloc(restart + 1, sizeof(double));
    double *y = calloc(restart, sizeof(double));
    orc_bilu0_apply(nf, bs, rowpts, colind, o2u, u2o, Mg, b, pb);
    const double nrmb = nrm2(N, pb);
    int iter = 0;
    *flag = 2;
    for (;;) {
        orc_matvec(nf, bs, rowpts, colind, Hg, x, t);
        orc_bilu0_apply(nf, bs, rowpts, colind, o2u, u2o, Mg, t, r);
        for (size_t q = 0; q < N; q++) r[q] = pb[q] - r[q];
        const double beta = nrm2(N, r);
        if (beta == 0.0) { *flag = 0; break; }
        for (size_t q = 0; q < N; q++) V[q] = r[q] / beta;
        for (int q = 0; q <= restart; q++) g[q] = 0.0;
        g[0] = beta;
        int jdone = 0, stop = 0;
        for (int j = 0; j < restart; j++) {
            double *vj = V + N * j, *w = V + N * (j + 1);
            orc_matvec(nf, bs, rowpts, colind, Hg, vj, t);
            orc_bilu0_apply(nf, bs, rowpts, colind, o2u, u2o, Mg, t, w);
            double *hc = Hh + (size_t)(restart + 1) * j;
            for (int i = 0; i <= j; i++) {
                const double *vi = V + N * i;
                double h = 0.0;
                for (size_t q = 0; q < N; q++) h += vi[q] * w[q];
                hc[i] = h;
                for (size_t q = 0; q < N; q++) w[q] -= h * vi[q];
            }
            hc[j + 1] = nrm2(N, w);
            if (hc[j + 1] == 0.0) { stop = 1; jdone = j; break; }
            for (size_t q = 0; q < N; q++) w[q] /= hc[j + 1];
            for (int i = 0; i < j; i++) {
                const double a = hc[i], bb = hc[i + 1];
                hc[i] = cs[i] * a + sn[i] * bb;
                hc[i + 1] = -sn[i] * a + cs[i] * bb;
            }
            const double a = hc[j], bb = hc[j + 1], den = sqrt(a * a + bb * bb);
            cs[j] = a / den; sn[j] = bb / den;
            hc[j] = den; hc[j + 1] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            const double res = fabs(g[j + 1]);
            if (rev) rev[iter] = res / nrmb;
            iter++;
            jdone = j + 1;
            if (res / nrmb <= tol) { *flag = 0; stop = 1; break; }
            if (iter >= maxit) { *flag = 1; stop = 1; break; }
        }
        const int m = jdone;
        for (int i = m - 1; i >= 0; i--) {
            double s = g[i];
            for (int l = i + 1; l < m; l++) s -= Hh[i + (size_t)(restart + 1) * l] * y[l];
            y[i] = s / Hh[i + (size_t)(restart + 1) * i];
        }
        for (int i = 0; i < m; i++) for (size_t q = 0; q < N; q++) x[q] += V[N * i + q] * y[i];
        if (stop) break;
    }
    free(pb); free(r); free(t); free(V); free(Hh); free(cs); free(sn); free(g); free(y);
    return iter;
}

/* hdg_solve.m:119-121: DUDGT = DUDG + DUDG_DUH * DUH(:, elcon(:,e)). */
void orc_backsub(int ne, int npv, int nc, int ncu, int ndf, const int *elcon, const double *DUDG,
                 const double *DUDG_DUH, const double *DUH, double *DUDGT)
{
    const int nq = npv * nc, nh = ncu * ndf;
    for (int e = 0; e < ne; e++) {
        const double *D = DUDG_DUH + (size_t)nq * nh * e;
        double *o = DUDGT + (size_t)nq * e;
        for (int q = 0; q < nq; q++) o[q] = DUDG[(size_t)nq * e + q];
        for (int f = 0; f < ndf; f++) {
            const int g = elcon[f + ndf * e] - 1;
            for (int c = 0; c < ncu; c++) {
                const double u = DUH[c + (size_t)ncu * g];
                const double *col = D + (size_t)nq * (c + ncu * f);
                for (int q = 0; q < nq; q++) o[q] += col[q] * u;
            }
        }
    }
}

/* ------------------------------------------------------------------ dense face-block path */

/* mesh/mkmesh/mkf2f.m + kernel/mkDenseBlockSystem.m:9-95 (mkBlockSystem1) restated from the
 * elemental arrays.  fel[2*nf]: the two elements of every face (1-based; <= 0 for none,
 * f(:,end-1:end)); t2f [ne, nfe] 1-based column-major; elcon [npf*nfe, ne] 1-based.
 * Outputs f2f [nbf, nf] (1-based, 0 = none), K [ncf, ncf*(nbf-1), nf], F [ncf, nf] with
 * ncf = ncu*npf, nbf = 2*nfe - 1.  The face blocks are read from AE with the face-local node
 * index j(n) = elcon(n, a, e) - (i-1)*npf used as an index into AE's face nodes, as
 * mkDenseBlockSystem.m:45-74 does (equal to the placement by elcon when j is its own
 * inverse, which holds for the two orientations of a 2D face).  Each block row is scaled
 * by inv(M) (mkDenseBlockSystem.m:90-94).  Returns the number of singular diagonal blocks. */
int orc_dense_block_system(int ne, int nfe, int npf, int ncu, int nf, const int *fel, const int *t2f,
                           const int *elcon, const double *AE, const double *FE, int *f2f, double *K, double *F)
{
    const int nbf = 2 * nfe - 1, ncf = ncu * npf, ndf = npf * nfe, nh = ncu * ndf, nn = nbf - 1;
    int nbad = 0;
    double *M = malloc(sizeof(double) * ncf * ncf), *T = malloc(sizeof(double) * ncf * ncf);
    int *j1 = malloc(sizeof(int) * npf), *j2 = malloc(sizeof(int) * npf), *j3 = malloc(sizeof(int) * npf);
    memset(f2f, 0, sizeof(int) * (size_t)nbf * nf);
    memset(K, 0, sizeof(double) * (size_t)ncf * ncf * nn * nf);
    /* AE(c, n, a, c2, n2, a2, e) with AE [ncu, npf, nfe, ncu, npf, nfe, ne] */
#define AEX(c, n, a, c2, n2, a2, e) AE[(c) + ncu * ((n) + npf * ((a) + nfe * ((size_t)(c2) + ncu * ((n2) + npf * ((a2) + (size_t)nfe * (e))))))]
    for (int i = 0; i < nf; i++) {
        const int e1 = fel[2 * i] - 1, e2 = fel[2 * i + 1] - 1;
        const int ne2 = e2 >= 0 ? 2 : 1;
        const int el[2] = {e1, e2};
        int fi[2] = {-1, -1};
        for (int q = 0; q < ne2; q++)
            for (int a = 0; a < nfe; a++)
                if (t2f[el[q] + ne * a] - 1 == i) { fi[q] = a; break; }
        for (int n = 0; n < npf; n++) j1[n] = elcon[n + npf * fi[0] + (size_t)ndf * e1] - 1 - i * npf;
        if (ne2 == 2)
            for (int n = 0; n < npf; n++) j2[n] = elcon[n + npf * fi[1] + (size_t)ndf * e2] - 1 - i * npf;
        f2f[nbf * i] = i + 1;
        for (int c = 0; c < ncu; c++)
            for (int n = 0; n < npf; n++) {
                double fv = FE[c + ncu * (j1[n] + npf * fi[0]) + (size_t)nh * e1];
                if (ne2 == 2) fv += FE[c + ncu * (j2[n] + npf * fi[1]) + (size_t)nh * e2];
                F[c + ncu * n + (size_t)ncf * i] = fv;
                for (int c2 = 0; c2 < ncu; c2++)
                    for (int n2 = 0; n2 < npf; n2++) {
                        double v = AEX(c, j1[n], fi[0], c2, j1[n2], fi[0], e1);
                        if (ne2 == 2) v += AEX(c, j2[n], fi[1], c2, j2[n2], fi[1], e2);
                        M[(c + ncu * n) + ncf * (c2 + ncu * n2)] = v;
                    }
            }
        int k = 0;
        for (int q = 0; q < ne2; q++) {
            const int e = el[q], ia = fi[q];
            const int *jq = q == 0 ? j1 : j2;
            for (int is = 0; is < nfe; is++) {
                if (is == ia) continue;
                const int jf = t2f[e + ne * is] - 1;
                f2f[(k + 1) + nbf * i] = jf + 1;
                for (int n = 0; n < npf; n++) j3[n] = elcon[n + npf * is + (size_t)ndf * e] - 1 - jf * npf;
                double *Kb = K + (size_t)ncf * ncf * (k + (size_t)nn * i);
                for (int c = 0; c < ncu; c++)
                    for (int n = 0; n < npf; n++)
                        for (int c2 = 0; c2 < ncu; c2++)
                            for (int n2 = 0; n2 < npf; n2++)
                                Kb[(c + ncu * n) + ncf * (c2 + ncu * n2)] = AEX(c, jq[n], ia, c2, j3[n2], is, e);
                k++;
            }
        }
        /* Mi = inv(M); F(:,i) = Mi F(:,i); K(:,:,j,i) = Mi K(:,:,j,i) */
        if (inv_inplace(ncf, M)) nbad++;
        double *fcol = F + (size_t)ncf * i, *tmp = T;
        for (int r = 0; r < ncf; r++) {
            double s = 0.0;
            for (int c = 0; c < ncf; c++) s += M[r + ncf * c] * fcol[c];
            tmp[r] = s;
        }
        memcpy(fcol, tmp, sizeof(double) * ncf);
        for (int q = 0; q < nn; q++) {
            double *Kb = K + (size_t)ncf * ncf * (q + (size_t)nn * i);
            mm(ncf, M, Kb, T);
            memcpy(Kb, T, sizeof(double) * ncf * ncf);
        }
    }
#undef AEX
    free(M); free(T); free(j1); free(j2); free(j3);
    return nbad;
}

/* kernel/gmres.m:40-44: y = x + K gather(x, f2f). */
void orc_dense_matvec(int nb, int nf, int nbf, const double *K, const int *f2f, const double *x, double *y)
{
    const int nn = nbf - 1;
    for (int i = 0; i < nf; i++)
        for (int r = 0; r < nb; r++) {
            double s = x[r + (size_t)nb * i];
            for (int k = 0; k < nn; k++) {
                const int j = f2f[(k + 1) + nbf * i];
                if (j <= 0) continue;
                const double *Kk = K + (size_t)nb * nb * (k + (size_t)nn * i);
                for (int c = 0; c < nb; c++) s += Kk[r + nb * c] * x[c + (size_t)nb * (j - 1)];
            }
            y[r + (size_t)nb * i] = s;
        }
}

/* kernel/gmres.m:1-111: unpreconditioned restarted GMRES on x + K gather(x) with classical
 * Gram-Schmidt (gmres.m:80-81); the least-squares problem of gmres.m:90 is solved with Givens
 * rotations (same minimiser and residual).  Iterations are counted as gmres.m counts them (the
 * residual evaluation at each restart is one).  Returns iterations; *flag 0 converged /
 * 1 maxit; rev[maxit] relative residuals (may be NULL). */
int orc_gmres_dense(int nb, int nf, int nbf, const double *K, const int *f2f, const double *b, double *x,
                    int restart, double tol, int maxit, int *flag, double *rev)
{
    const size_t N = (size_t)nb * nf;
    double *t = malloc(sizeof(double) * N), *V = malloc(sizeof(double) * N * (restart + 1));
    double *Hh = calloc((size_t)(restart + 1) * restart, sizeof(double));
    double *cs = calloc(restart, sizeof(double)), *sn = calloc(restart, sizeof(double));
    double *g = calloc(restart + 1, sizeof(double)), *y = calloc(restart, sizeof(double));
    const double nrmb = nrm2(N, b);
    int iter = 0;
    *flag = 2;
    if (!(nrmb > 0.0)) *flag = 0;
    while (*flag == 2) {
        orc_dense_matvec(nb, nf, nbf, K, f2f, x, t);
        for (size_t q = 0; q < N; q++) V[q] = b[q] - t[q];
        const double beta = nrm2(N, V);
        double res = beta;
        if (rev && iter < maxit) rev[iter] = res / nrmb;
        iter++;
        if (res / nrmb <= tol) { *flag = 0; break; }
        if (iter >= maxit) { *flag = 1; break; }
        for (size_t q = 0; q < N; q++) V[q] /= beta;
        for (int q = 0; q <= restart; q++) g[q] = 0.0;
        g[0] = beta;
        int jdone = 0;
        for (int j = 0; j < restart; j++) {
            if (j > 0) {
                if (res / nrmb <= tol) { *flag = 0; break; }
                if (iter >= maxit) { *flag = 1; break; }
            }
            double *w = V + N * (j + 1), *hc = Hh + (size_t)(restart + 1) * j;
            orc_dense_matvec(nb, nf, nbf, K, f2f, V + N * j, w);
            for (int i = 0; i <= j; i++) {             /* h = V' w with the unmodified w */
                const double *vi = V + N * i;
                double h = 0.0;
                for (size_t q = 0; q < N; q++) h += vi[q] * w[q];
                hc[i] = h;
            }
            for (int i = 0; i <= j; i++) {
                const double *vi = V + N * i;
                for (size_t q = 0; q < N; q++) w[q] -= hc[i] * vi[q];
            }
            hc[j + 1] = nrm2(N, w);
            const double sub = hc[j + 1];
            if (sub != 0.0) for (size_t q = 0; q < N; q++) w[q] /= sub;
            for (int i = 0; i < j; i++) {
                const double a = hc[i], bb = hc[i + 1];
                hc[i] = cs[i] * a + sn[i] * bb;
                hc[i + 1] = -sn[i] * a + cs[i] * bb;
            }
            const double a = hc[j], bb = hc[j + 1], den = sqrt(a * a + bb * bb);
            cs[j] = den != 0.0 ? a / den : 1.0; sn[j] = den != 0.0 ? bb / den : 0.0;
            hc[j] = den; hc[j + 1] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            res = fabs(g[j + 1]);
            if (rev && iter < maxit) rev[iter] = res / nrmb;
            iter++;
            jdone = j + 1;
            if (sub == 0.0) break;
        }
        for (int i = jdone - 1; i >= 0; i--) {
            double s = g[i];
            for (int l = i + 1; l < jdone; l++) s -= Hh[i + (size_t)(restart + 1) * l] * y[l];
            y[i] = s / Hh[i + (size_t)(restart + 1) * i];
        }
        for (int i = 0; i < jdone; i++) for (size_t q = 0; q < N; q++) x[q] += V[N * i + q] * y[i];
    }
    free(t); free(V); free(Hh); free(cs); free(sn); free(g); free(y);
    return iter;
}
