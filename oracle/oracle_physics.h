/*
 * oracle_physics.h -- CPU restatement of the compressible Navier-Stokes / Euler point
 * functions of the reference (TEST INFRASTRUCTURE: only tests/, the smoke check and the
 * CPU baseline of bench.py use anything under oracle/).
 *
 * Follows:
 *   flux : application/FM/ns/flux2d.m:27-126 (3D: flux3d.m); the generated C twins
 *          application/FM/ns/flux_ns2d.c / flux_ns3d.c compute the same expressions.
 *          f_x = [ru, ru u + p + txx, rv u + txy, (rE+p) u + u txx + v txy + kap d_x(p/r)]
 *          where q = (gradient slots of udg) stands for grad(u) as written in the reference
 *          (its sign convention is q = -grad u), txx = (1/Re)(2 u_x - 2/3 div), txy =
 *          (1/Re)(u_y + v_x), kap = gam / (Re Pr (gam-1)).  Euler = the same with 1/Re = 0.
 *   fhat : application/FM/ns/fhat.m:49-67  fh = f(uh, q) . n + tau (u - uh)
 *   fbou : application/FM/ns/fbou.m:111-114 (ib 6, Dirichlet: fh = uh - uinf),
 *          fbou.m case 5 (periodic: fhat).
 * Jacobians are computed exactly by forward-mode differentiation (value + nc partials).
 * param = {gam, epslm, Re, Pr, Minf, tau} (problem/ns/ns_naca.m:36).
 */
#ifndef ORACLE_PHYSICS_H
#define ORACLE_PHYSICS_H

#define ORC_MAXD 20

typedef struct { double v; double d[ORC_MAXD]; } odual;

static inline odual od_c(double v, int n) { odual r; r.v = v; for (int i = 0; i < n; i++) r.d[i] = 0.0; return r; }
static inline odual od_var(double v, int k, int n) { odual r = od_c(v, n); r.d[k] = 1.0; return r; }
static inline odual od_add(odual a, odual b, int n) { odual r; r.v = a.v + b.v; for (int i = 0; i < n; i++) r.d[i] = a.d[i] + b.d[i]; return r; }
static inline odual od_sub(odual a, odual b, int n) { odual r; r.v = a.v - b.v; for (int i = 0; i < n; i++) r.d[i] = a.d[i] - b.d[i]; return r; }
static inline odual od_mul(odual a, odual b, int n) { odual r; r.v = a.v * b.v; for (int i = 0; i < n; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i]; return r; }
static inline odual od_scale(odual a, double s, int n) { odual r; r.v = a.v * s; for (int i = 0; i < n; i++) r.d[i] = a.d[i] * s; return r; }
static inline odual od_div(odual a, odual b, int n) {
    odual r; double ib = 1.0 / b.v; r.v = a.v * ib;
    for (int i = 0; i < n; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}

/* f[a + ncu*j] and df[a + ncu*j][c] for one point: x-direction j flux of component a.
 * u[ncu] conserved state, q[ncu*nd] gradient slots (component fastest), all as duals. */
static void orc_ns_point(int nd, const double *param, const odual *u, const odual *q, int n,
                         odual *f /* [ncu*nd] */)
{
    const int ncu = nd + 2;
    const double gam = param[0], gam1 = param[0] - 1.0;
    const double rinv = 1.0 / param[2];                 /* 1/Re (0 for Euler, Re = inf) */
    const double kap = gam * rinv / (param[3] * gam1);  /* gam/(Re Pr (gam-1)) */
    odual r = u[0], rE = u[ncu - 1];
    odual vel[3], mom[3];
    odual ke = od_c(0.0, n);
    for (int i = 0; i < nd; i++) {
        mom[i] = u[1 + i];
        vel[i] = od_div(mom[i], r, n);
        ke = od_add(ke, od_mul(vel[i], mom[i], n), n);
    }
    ke = od_scale(ke, 0.5, n);                            /* r |v|^2 / 2 */
    odual p = od_scale(od_sub(rE, ke, n), gam1, n);
    /* velocity gradient from q: dv_i/dx_j = (q_{mom_i,j} - v_i q_{r,j}) / r */
    odual gv[3][3];
    for (int i = 0; i < nd; i++)
        for (int j = 0; j < nd; j++)
            gv[i][j] = od_div(od_sub(q[(1 + i) + ncu * j], od_mul(vel[i], q[0 + ncu * j], n), n), r, n);
    odual div = od_c(0.0, n);
    for (int i = 0; i < nd; i++) div = od_add(div, gv[i][i], n);
    odual tau[3][3];
    for (int i = 0; i < nd; i++)
        for (int j = 0; j < nd; j++) {
            odual t = od_add(gv[i][j], gv[j][i], n);
            if (i == j) t = od_sub(t, od_scale(div, 2.0 / 3.0, n), n);
            tau[i][j] = od_scale(t, rinv, n);
        }
    /* d_j(p/r) from q: p_j = gam1 (q_{rE,j} - 1/2 |v|^2 q_{r,j} - r v . v_j) */
    odual v2 = od_c(0.0, n);
    for (int i = 0; i < nd; i++) v2 = od_add(v2, od_mul(vel[i], vel[i], n), n);
    odual h = od_div(od_add(rE, p, n), r, n);
    for (int j = 0; j < nd; j++) {
        odual vdv = od_c(0.0, n);
        for (int i = 0; i < nd; i++) vdv = od_add(vdv, od_mul(vel[i], gv[i][j], n), n);
        odual pj = od_sub(od_sub(q[(ncu - 1) + ncu * j], od_mul(od_scale(v2, 0.5, n), q[0 + ncu * j], n), n),
                          od_mul(r, vdv, n), n);
        pj = od_scale(pj, gam1, n);
        odual Tj = od_div(od_sub(od_mul(pj, r, n), od_mul(p, q[0 + ncu * j], n), n), od_mul(r, r, n), n);
        f[0 + ncu * j] = mom[j];
        for (int i = 0; i < nd; i++) {
            odual t = od_add(od_mul(mom[i], vel[j], n), tau[i][j], n);
            if (i == j) t = od_add(t, p, n);
            f[(1 + i) + ncu * j] = t;
        }
        odual e = od_mul(h, mom[j], n);
        for (int i = 0; i < nd; i++) e = od_add(e, od_mul(vel[i], tau[i][j], n), n);
        e = od_add(e, od_scale(Tj, kap, n), n);
        f[(ncu - 1) + ncu * j] = e;
    }
}

/* Volume flux (flux.m layout): f[ng,ncu,nd], f_udg[ng,ncu,nd,nc]; udg[ng,nc]. */
static void orc_flux(int nd, const double *param, int ng, const double *udg, double *f, double *f_udg)
{
    const int ncu = nd + 2, nc = ncu * (nd + 1);
    for (int g = 0; g < ng; g++) {
        odual u[5], q[15], ff[15];
        for (int c = 0; c < ncu; c++) u[c] = od_var(udg[g + ng * c], c, nc);
        for (int c = 0; c < ncu * nd; c++) q[c] = od_var(udg[g + ng * (ncu + c)], ncu + c, nc);
        orc_ns_point(nd, param, u, q, nc, ff);
        for (int j = 0; j < nd; j++)
            for (int a = 0; a < ncu; a++) {
                const odual *x = &ff[a + ncu * j];
                f[g + ng * (a + ncu * j)] = x->v;
                for (int c = 0; c < nc; c++)
                    f_udg[g + ng * (a + ncu * (j + nd * c))] = x->d[c];
            }
    }
}

/* Numerical trace flux (fhat.m): fh[ng,ncu], fh_udg[ng,ncu,nc], fh_uh[ng,ncu,ncu]. */
static void orc_fhat(int nd, const double *param, int ng, const double *nl, const double *udg,
                     const double *uh, double *fh, double *fh_udg, double *fh_uh)
{
    const int ncu = nd + 2, nc = ncu * (nd + 1);
    const double tau = param[5];
    for (int g = 0; g < ng; g++) {
        odual u[5], q[15], ff[15];
        for (int c = 0; c < ncu; c++) u[c] = od_var(uh[g + ng * c], c, nc);
        for (int c = 0; c < ncu * nd; c++) q[c] = od_var(udg[g + ng * (ncu + c)], ncu + c, nc);
        orc_ns_point(nd, param, u, q, nc, ff);
        for (int a = 0; a < ncu; a++) {
            double v = 0.0, dv[ORC_MAXD];
            for (int c = 0; c < nc; c++) dv[c] = 0.0;
            for (int j = 0; j < nd; j++) {
                double nj = nl[g + ng * j];
                v += ff[a + ncu * j].v * nj;
                for (int c = 0; c < nc; c++) dv[c] += ff[a + ncu * j].d[c] * nj;
            }
            fh[g + ng * a] = v + tau * (udg[g + ng * a] - uh[g + ng * a]);
            for (int c = 0; c < nc; c++)
                fh_udg[g + ng * (a + ncu * c)] = (c < ncu) ? ((c == a) ? tau : 0.0) : dv[c];
            for (int b = 0; b < ncu; b++)
                fh_uh[g + ng * (a + ncu * b)] = dv[b] - ((a == b) ? tau : 0.0);
        }
    }
}

/* Boundary flux (fbou.m): ib 6 Dirichlet fh = uh - uinf; ib 5 periodic = fhat.
 * Returns 0 on success, -1 for a boundary type this restatement does not cover. */
static int orc_fbou(int nd, int ib, const double *uinf, const double *param, int ng,
                    const double *nl, const double *udg, const double *uh,
                    double *fh, double *fh_udg, double *fh_uh)
{
    const int ncu = nd + 2, nc = ncu * (nd + 1);
    if (ib == 5) { orc_fhat(nd, param, ng, nl, udg, uh, fh, fh_udg, fh_uh); return 0; }
    if (ib != 6) return -1;
    for (int g = 0; g < ng; g++)
        for (int a = 0; a < ncu; a++) {
            fh[g + ng * a] = uh[g + ng * a] - uinf[a];
            for (int c = 0; c < nc; c++) fh_udg[g + ng * (a + ncu * c)] = 0.0;
            for (int b = 0; b < ncu; b++) fh_uh[g + ng * (a + ncu * b)] = (a == b) ? 1.0 : 0.0;
        }
    return 0;
}

#endif
