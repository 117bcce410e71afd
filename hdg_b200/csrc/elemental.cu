// elemental.cu -- dispatch of the fused elemental kernel (elemental_kernel.cuh): the compiled
// shapes by (nd, porder), the master check, the parameter block of a launch and the segmented
// launch over several element sets.  The launchers themselves are instantiated, shape by shape, in
// elemental_inst_*.cu so that the shapes compile in parallel.
#include "elemental_kernel.cuh"

HDGX_ELEM_LAUNCHERS(extern, hdgx::Tri1)
HDGX_ELEM_LAUNCHERS(extern, hdgx::Tri2)
HDGX_ELEM_LAUNCHERS(extern, hdgx::Tri3)
HDGX_ELEM_LAUNCHERS(extern, hdgx::Tri4)
HDGX_ELEM_LAUNCHERS(extern, hdgx::Tet1)
HDGX_ELEM_LAUNCHERS(extern, hdgx::Tet2)
HDGX_ELEM_LAUNCHERS_FP64(extern, hdgx::Tet3)

namespace hdgx {

template <class D>
static int launch_v(const ElemParams &p, bool visc, bool mixed, cudaStream_t st, int grid) {
    if constexpr (PlanSel<D, true, false>::WS || PlanSel<D, false, false>::WS) {
        // plans in the global workspace are built in FP64 only: the mixed form runs the FP64 kernel
        return visc ? launch_t<D, true, false>(p, p.ne, st, grid) : launch_t<D, false, false>(p, p.ne, st, grid);
    } else {
        if (mixed)
            return visc ? launch_t<D, true, true>(p, p.ne, st, grid) : launch_t<D, false, true>(p, p.ne, st, grid);
        return visc ? launch_t<D, true, false>(p, p.ne, st, grid) : launch_t<D, false, false>(p, p.ne, st, grid);
    }
}

// The compiled element shapes, keyed by (nd, porder).  Their Gauss point counts are those of
// the drivers' quadrature order pgauss = 2 porder (mkmaster(mesh, 2*porder), e.g.
// problem/euler/euler_trefftz.m:55); f(Dims{}) is called for the match, -3 returned otherwise.
template <class F>
static int with_dims(int nd, int po, F &&f) {
    if (nd == 2) {
        switch (po) {
            case 1: return f(Tri1{});
            case 2: return f(Tri2{});
            case 3: return f(Tri3{});
            case 4: return f(Tri4{});
        }
    } else if (nd == 3) {
        switch (po) {
            case 1: return f(Tet1{});
            case 2: return f(Tet2{});
            case 3: return f(Tet3{});
        }
    }
    return -3;
}

// 0 when the master's table sizes are those of the compiled kernel for its (nd, porder), -3
// otherwise.  mkmaster(mesh, pgauss) (master/mkmaster.m:1) takes the quadrature order as a
// free argument; a master built with pgauss != 2 porder has other ngv / ngf, and the kernel,
// whose loops run over the compiled extents, would index its tables out of range.
int elemental_check_master(const hdgx_master *m) {
    if (!m) return -1;
    return with_dims(m->nd, m->porder, [&](auto d) -> int {
        using D = decltype(d);
        const bool ok = m->npv == D::NPV && m->npf == D::NPF && m->ngv == D::NGV && m->ngf == D::NGF &&
                        m->nfe == D::NFE;
        return ok ? 0 : -3;
    });
}

static ElemParams fill_params(const hdgx_master *m, const hdgx_app *app, int ne, const double *dgnodes,
                              const int *bf, const double *UDG, const double *UH, const double *SH, double *AE,
                              double *FE, double *DUDG, double *DUDG_DUH, int *status, double *QDG, double *RU) {
    ElemParams p;
    p.shapvt = m->shapvt; p.shapvg = m->shapvg; p.shapmv = m->shapmv;
    p.shapft = m->shapft; p.shapfg = m->shapfg; p.shapmf = m->shapmf; p.perm = m->perm;
    const double gam = app->param[0], re = app->param[2], pr = app->param[3];
    p.pc.gam1 = gam - 1.0;
    p.pc.rinv = (re > 0.0 && isfinite(re)) ? 1.0 / re : 0.0;
    p.pc.kap = p.pc.rinv * gam / (pr * (gam - 1.0));
    p.pc.tau = app->param[5];
    p.fb.fam = app->fbou;
    p.fb.gam = gam;
    p.fb.eps = app->param[1];
    p.fb.m2 = app->param[4] * app->param[4];
    p.fc_q = app->fc_q;
    p.fc_u = app->fc_u;
    p.tdep = app->tdep;
    p.nbnd = app->nbnd;
    for (int i = 0; i < HDGX_MAX_BND; i++) p.bcm[i] = app->bcm[i];
    for (int i = 0; i < HDGX_MAX_BND * 5; i++) p.bcs[i] = app->bcs[i];
    p.ne = ne; p.dgnodes = dgnodes; p.UDG = UDG; p.UH = UH; p.SH = SH; p.bf = bf;
    p.AE = AE; p.FE = FE; p.DUDG = DUDG; p.DUDG_DUH = DUDG_DUH; p.status = status;
    p.QDG = QDG;
    p.RU = RU;
    p.nco = app->getdqdg ? app->nc : app->ncu;
    p.ws = nullptr;
    return p;
}

static bool is_viscous(const hdgx_app *app) {
    const double re = app->param[2];
    return re > 0.0 && isfinite(re);
}

int elemental_launch(const hdgx_master *m, const hdgx_app *app, int ne, const double *dgnodes,
                     const int *bf, const double *UDG, const double *UH, const double *SH, double *AE,
                     double *FE, double *DUDG, double *DUDG_DUH, int *status, cudaStream_t st, bool mixed,
                     int grid, double *QDG, double *RU) {
    const ElemParams p = fill_params(m, app, ne, dgnodes, bf, UDG, UH, SH, AE, FE, DUDG, DUDG_DUH, status, QDG, RU);
    if (int rc = elemental_check_master(m)) return rc;   // nothing is launched for a foreign master
    return with_dims(m->nd, m->porder, [&](auto d) -> int {
        return launch_v<decltype(d)>(p, is_viscous(app), mixed, st, grid);
    });
}

int elemental_shared_max_segments() { return kMaxSeg; }

// One FP64 launch over the buckets' elements (callers have validated every bucket).  The buckets
// must have one element shape (nd, porder and the master's table sizes) and agree on whether the
// physics is viscous, which selects the kernel; each keeps its own app (physics constants,
// boundary data, getdqdg) and arrays.  The master tables are read from bucket 0's master.
int elemental_launch_shared(int nb, const hdgx_elem_bucket *b, cudaStream_t st, int grid) {
    if (nb < 1 || nb > kMaxSeg) return -1;
    const hdgx_master *m0 = b[0].master;
    const bool visc = is_viscous(b[0].app);
    for (int k = 1; k < nb; k++) {
        const hdgx_master *m = b[k].master;
        if (m->nd != m0->nd || m->porder != m0->porder || m->npv != m0->npv || m->npf != m0->npf ||
            m->ngv != m0->ngv || m->ngf != m0->ngf)
            return -2;
        if (is_viscous(b[k].app) != visc) return -2;
    }
    if (int rc = elemental_check_master(m0)) return rc;
    SegTable t;
    int n = 0;
    for (int k = 0; k < nb; k++) {
        const hdgx_elem_bucket &q = b[k];
        t.seg[k] = fill_params(m0, q.app, q.ne, q.dgnodes, q.bf, q.UDG, q.UH, q.SH, q.AE, q.FE, q.DUDG, q.DUDG_DUH,
                               q.status, nullptr, nullptr);
        t.seg_start[k] = n;
        n += q.ne;
    }
    t.seg_start[nb] = n;
    t.nseg = nb;
    if (n == 0) return 0;
    return with_dims(m0->nd, m0->porder, [&](auto d) -> int {
        using D = decltype(d);
        return visc ? launch_t<D, true, false>(t, n, st, grid) : launch_t<D, false, false>(t, n, st, grid);
    });
}

}  // namespace hdgx
