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
 *   fbou : two families, as the app's physics folder selects them (faceint.m:171-268 calls
 *          app.fbou of application/FM/<physics>):
 *          ns    application/FM/ns/fbou.m (fbou3d.m in 3D): 1 far field through the Roe
 *                matrices of getan.m / getan3d.m (application/FM/getan.c), 2 adiabatic wall,
 *                3 isothermal wall, 4 prescribed pressure, 5 periodic (fhat), 6 Dirichlet
 *                fh = uh - uinf (fbou.m:111-114);
 *          euler application/FM/euler/fbou.m: 1 far field with the local Lax-Friedrichs
 *                scalars of euler/getan.m (absolute 2 / 3), 2 slip wall, 3 and 4 prescribed
 *                pressure, 5 density and energy extrapolated; 6 Dirichlet as the ns family.
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

static inline odual od_sqrt(odual a, int n) {
    odual r; r.v = sqrt(a.v);
    const double h = 0.5 / r.v;
    for (int i = 0; i < n; i++) r.d[i] = a.d[i] * h;
    return r;
}
/* |a| with the derivative sign(a) a' (sign(0) = 1) */
static inline odual od_abs(odual a, int n) { return a.v < 0.0 ? od_scale(a, -1.0, n) : a; }

/* Sound speed c, normal velocity un, velocity v[nd], kinetic energy per mass af = |v|^2/2 and
 * total enthalpy h of the conserved state m[ncu] (the quantities getan.m forms first). */
static void orc_state(int nd, double gam, const odual *m, const double *nl, int n,
                      odual *c, odual *un, odual *v, odual *af, odual *h)
{
    const int ncu = nd + 2;
    const double gam1 = gam - 1.0;
    odual r = m[0];
    *un = od_c(0.0, n);
    *af = od_c(0.0, n);
    for (int i = 0; i < nd; i++) {
        v[i] = od_div(m[1 + i], r, n);
        *un = od_add(*un, od_scale(v[i], nl[i], n), n);
        *af = od_add(*af, od_scale(od_mul(v[i], v[i], n), 0.5, n), n);
    }
    odual p = od_scale(od_sub(m[ncu - 1], od_mul(r, *af, n), n), gam1, n);
    *c = od_sqrt(od_div(od_scale(p, gam, n), r, n), n);
    *h = od_div(od_add(m[ncu - 1], p, n), r, n);
}

/* The Roe matrices of application/FM/ns/getan.m (getan3d.m; the generated twin is
 * application/FM/getan.c): absolute 0 gives the normal flux Jacobian A_n(m), absolute 1 its
 * absolute value |A_n(m)|, both as the sum of the eigenvalue l3 = un times the identity and
 * two rank-one terms,
 *     An = l3 I + r1 w1' + r2 w2',   r1 = [1, v, h],  r2 = [0, n, un],
 *     w1 = (s1 - l3) gam1/c^2 P + s2/c N,  w2 = s2 gam1/c P + (s1 - l3) N,
 *     P = [af, -v, 1],  N = [-un, n, 0],  s1 = (l1 + l2)/2,  s2 = (l1 - l2)/2,
 * with l1 = un + c, l2 = un - c; for absolute 1 every l is replaced by |l| and, when
 * eps = param[1] > 0, by (|l|^2/(eps c) + eps c)/2 where |l| < eps c (getan.m:232-311).
 * An[j + ncu*k], derivatives with respect to whatever m carries. */
static void orc_getan_roe(int nd, const double *param, const double *nl, const odual *m, int absolute, int n,
                          odual *An)
{
    const int ncu = nd + 2;
    const double gam = param[0], gam1 = gam - 1.0, eps = param[1];
    odual c, un, v[3], af, h;
    orc_state(nd, gam, m, nl, n, &c, &un, v, &af, &h);
    odual l[3] = {od_add(un, c, n), od_sub(un, c, n), un};
    if (absolute) {
        odual ec = od_scale(c, eps, n);
        for (int i = 0; i < 3; i++) {
            l[i] = od_abs(l[i], n);
            if (eps > 0.0 && l[i].v < ec.v)
                l[i] = od_scale(od_add(od_div(od_mul(l[i], l[i], n), ec, n), ec, n), 0.5, n);
        }
    }
    odual s1 = od_scale(od_add(l[0], l[1], n), 0.5, n), s2 = od_scale(od_sub(l[0], l[1], n), 0.5, n);
    odual d = od_sub(s1, l[2], n);
    odual k1 = od_div(od_scale(d, gam1, n), od_mul(c, c, n), n);     /* (s1 - l3) gam1 / c^2 */
    odual k2 = od_div(s2, c, n);                                    /* s2 / c */
    odual k3 = od_scale(k2, gam1, n);                               /* s2 gam1 / c */
    odual r1[5], r2[5], P[5], N[5];
    r1[0] = od_c(1.0, n); r2[0] = od_c(0.0, n); P[0] = af; N[0] = od_scale(un, -1.0, n);
    for (int i = 0; i < nd; i++) {
        r1[1 + i] = v[i]; r2[1 + i] = od_c(nl[i], n);
        P[1 + i] = od_scale(v[i], -1.0, n); N[1 + i] = od_c(nl[i], n);
    }
    r1[ncu - 1] = h; r2[ncu - 1] = un; P[ncu - 1] = od_c(1.0, n); N[ncu - 1] = od_c(0.0, n);
    for (int k = 0; k < ncu; k++) {
        odual w1 = od_add(od_mul(k1, P[k], n), od_mul(k2, N[k], n), n);
        odual w2 = od_add(od_mul(k3, P[k], n), od_mul(d, N[k], n), n);
        for (int j = 0; j < ncu; j++) {
            odual t = od_add(od_mul(r1[j], w1, n), od_mul(r2[j], w2, n), n);
            if (j == k) t = od_add(t, l[2], n);
            An[j + ncu * k] = t;
        }
    }
}

/* The local Lax-Friedrichs scalars of application/FM/euler/getan.m:25-111 at the state m:
 * absolute 2 gives |un| + c (with eps = param[1] > 0: ((|un| + c)^2/(eps c) + eps c)/2),
 * absolute 3 gives un - c.  Both multiply the identity there. */
static odual orc_getan_llf(int nd, const double *param, const double *nl, const odual *m, int absolute, int n)
{
    const double gam = param[0], eps = param[1];
    odual c, un, v[3], af, h;
    orc_state(nd, gam, m, nl, n, &c, &un, v, &af, &h);
    if (absolute == 3) return od_sub(un, c, n);
    odual lam = od_add(od_abs(un, n), c, n);
    if (eps > 0.0) {
        odual ec = od_scale(c, eps, n);
        lam = od_scale(od_add(od_div(od_mul(lam, lam, n), ec, n), ec, n), 0.5, n);
    }
    return lam;
}

/* uinf with the energy set from the pressure p and the interior density and momentum:
 * [u0, u_mom, p/(gam-1) + |u_mom|^2/(2 u0)] (euler/fbou.m:52,64; ns/fbou.m:97) */
static void orc_pressure_state(int nd, double gam, double p, const odual *u, int n, odual *uinf)
{
    const int ncu = nd + 2;
    odual ke = od_c(0.0, n);
    for (int i = 0; i < nd; i++) {
        uinf[1 + i] = u[1 + i];
        ke = od_add(ke, od_div(od_mul(u[1 + i], u[1 + i], n), u[0], n), n);
    }
    uinf[0] = u[0];
    uinf[ncu - 1] = od_add(od_c(p / (gam - 1.0), n), od_scale(ke, 0.5, n), n);
}

/* One point of fbou: fh[ncu] from the interior state u[ncu], its gradient slots q[ncu*nd], the
 * trace uh[ncu], the boundary state ub[ncu] (the row bcs(ib, :)) and the unit normal nl[nd].
 * fam 0: application/FM/ns/fbou.m (fbou3d.m), fam 1: application/FM/euler/fbou.m.
 * Returns 0, or -1 for a type this restatement does not cover. */
static int orc_fbou_point(int fam, int nd, int ib, const double *ub, const double *param, const double *nl,
                          const odual *u, const odual *q, const odual *uh, int n, odual *fh)
{
    const int ncu = nd + 2;
    const double gam = param[0], gam1 = gam - 1.0;
    if (ib == 6) {                                         /* ns/fbou.m:111-114 */
        for (int a = 0; a < ncu; a++) fh[a] = od_sub(uh[a], od_c(ub[a], n), n);
        return 0;
    }
    odual uinf[5];
    if (fam == 0) {
        const double tau = param[5], minf = param[4];
        switch (ib) {
            case 1:                                        /* ns/fbou.m:37-46 */
            case 4: {                                      /* ns/fbou.m:93-108 */
                if (ib == 1)
                    for (int a = 0; a < ncu; a++) uinf[a] = od_c(ub[a], n);
                else
                    orc_pressure_state(nd, gam, (ub[ncu - 1] - 0.5) * gam1, u, n, uinf);
                odual an[25], An[25];
                orc_getan_roe(nd, param, nl, uh, 0, n, an);
                orc_getan_roe(nd, param, nl, uh, 1, n, An);
                for (int j = 0; j < ncu; j++) {
                    odual t = od_c(0.0, n);
                    for (int k = 0; k < ncu; k++) {
                        const odual p = od_add(an[j + ncu * k], An[j + ncu * k], n);
                        const odual m = od_sub(an[j + ncu * k], An[j + ncu * k], n);
                        t = od_add(t, od_mul(p, od_sub(u[k], uh[k], n), n), n);
                        t = od_sub(t, od_mul(m, od_sub(uinf[k], uh[k], n), n), n);
                    }
                    fh[j] = t;
                }
                return 0;
            }
            case 2:                                        /* ns/fbou.m:47-69, fbou3d.m:36-61 */
            case 3: {                                      /* ns/fbou.m:70-92, fbou3d.m:62-81 */
                fh[0] = od_sub(u[0], uh[0], n);
                for (int i = 0; i < nd; i++) fh[1 + i] = od_scale(uh[1 + i], -1.0, n);
                if (ib == 3) {
                    fh[ncu - 1] = od_sub(od_scale(od_div(uh[ncu - 1], uh[0], n), gam * gam1 * minf * minf, n),
                                         od_c(ub[ncu - 1], n), n);
                } else {
                    odual ff[15];                              /* the energy row of fhat */
                    orc_ns_point(nd, param, uh, q, n, ff);
                    odual e = od_scale(od_sub(u[ncu - 1], uh[ncu - 1], n), tau, n);
                    for (int j = 0; j < nd; j++) e = od_add(e, od_scale(ff[(ncu - 1) + ncu * j], nl[j], n), n);
                    fh[ncu - 1] = e;
                }
                return 0;
            }
            case 5: {                                      /* periodic: fhat (ns/fbou.m:109-110) */
                odual ff[15];
                orc_ns_point(nd, param, uh, q, n, ff);
                for (int a = 0; a < ncu; a++) {
                    odual e = od_scale(od_sub(u[a], uh[a], n), tau, n);
                    for (int j = 0; j < nd; j++) e = od_add(e, od_scale(ff[a + ncu * j], nl[j], n), n);
                    fh[a] = e;
                }
                return 0;
            }
        }
        return -1;
    }
    switch (ib) {
        case 1:                                            /* euler/fbou.m:24-29 */
        case 3:                                            /* euler/fbou.m:50-60 */
        case 4: {                                          /* euler/fbou.m:62-72 */
            if (ib == 1)
                for (int a = 0; a < ncu; a++) uinf[a] = od_c(ub[a], n);
            else
                orc_pressure_state(nd, gam, ib == 3 ? ub[0] : (ub[ncu - 1] - 0.5) * gam1, u, n, uinf);
            const odual an = orc_getan_llf(nd, param, nl, uh, 2, n), An = orc_getan_llf(nd, param, nl, uh, 3, n);
            const odual p = od_add(an, An, n), m = od_sub(an, An, n);
            for (int a = 0; a < ncu; a++)
                fh[a] = od_sub(od_mul(p, od_sub(u[a], uh[a], n), n), od_mul(m, od_sub(uinf[a], uh[a], n), n), n);
            return 0;
        }
        case 2: {                                          /* euler/fbou.m:30-48 */
            odual un = od_c(0.0, n);
            for (int i = 0; i < nd; i++) un = od_add(un, od_scale(u[1 + i], nl[i], n), n);
            fh[0] = od_sub(u[0], uh[0], n);
            for (int i = 0; i < nd; i++)
                fh[1 + i] = od_sub(od_sub(u[1 + i], od_scale(un, nl[i], n), n), uh[1 + i], n);
            fh[ncu - 1] = od_sub(u[ncu - 1], uh[ncu - 1], n);
            return 0;
        }
        case 5:                                            /* euler/fbou.m:73-87 */
            for (int a = 0; a < ncu; a++) {
                const odual b = (a == 0 || a == ncu - 1) ? u[a] : od_c(ub[a], n);
                fh[a] = od_sub(b, uh[a], n);
            }
            return 0;
    }
    return -1;
}

/* Boundary flux of family fam (0: ns/fbou.m, 1: euler/fbou.m) over ng points:
 * fh[ng,ncu], fh_udg[ng,ncu,nc], fh_uh[ng,ncu,ncu] from udg[ng,nc], uh[ng,ncu], nl[ng,nd].
 * Returns 0 on success, -1 for a boundary type this restatement does not cover. */
static int orc_fbou(int fam, int nd, int ib, const double *uinf, const double *param, int ng,
                    const double *nl, const double *udg, const double *uh,
                    double *fh, double *fh_udg, double *fh_uh)
{
    const int ncu = nd + 2, nc = ncu * (nd + 1);
    if (ib == 5 && fam == 0) { orc_fhat(nd, param, ng, nl, udg, uh, fh, fh_udg, fh_uh); return 0; }
    for (int g = 0; g < ng; g++) {
        double n1[3];
        for (int d = 0; d < nd; d++) n1[d] = nl[g + ng * d];
        odual u[5], q[15], h[5], f[5];
        /* derivatives with respect to (u, q) */
        for (int c = 0; c < ncu; c++) u[c] = od_var(udg[g + ng * c], c, nc);
        for (int c = 0; c < ncu * nd; c++) q[c] = od_var(udg[g + ng * (ncu + c)], ncu + c, nc);
        for (int c = 0; c < ncu; c++) h[c] = od_c(uh[g + ng * c], nc);
        if (orc_fbou_point(fam, nd, ib, uinf, param, n1, u, q, h, nc, f)) return -1;
        for (int a = 0; a < ncu; a++) {
            fh[g + ng * a] = f[a].v;
            for (int c = 0; c < nc; c++) fh_udg[g + ng * (a + ncu * c)] = f[a].d[c];
        }
        /* derivatives with respect to uh */
        for (int c = 0; c < ncu; c++) u[c] = od_c(udg[g + ng * c], ncu);
        for (int c = 0; c < ncu * nd; c++) q[c] = od_c(udg[g + ng * (ncu + c)], ncu);
        for (int c = 0; c < ncu; c++) h[c] = od_var(uh[g + ng * c], c, ncu);
        orc_fbou_point(fam, nd, ib, uinf, param, n1, u, q, h, ncu, f);
        for (int a = 0; a < ncu; a++)
            for (int b = 0; b < ncu; b++) fh_uh[g + ng * (a + ncu * b)] = f[a].d[b];
    }
    return 0;
}

#endif
