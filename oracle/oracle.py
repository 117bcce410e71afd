"""ctypes bindings of the CPU oracle (liboracle.so) and of the reference's compiled C
sources (oracle/_ref).  TEST INFRASTRUCTURE: only tests/, the smoke check and bench.py's
CPU baseline leg import this module; the product never does."""
from __future__ import annotations

import ctypes as ct
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = None
_REF = {}

_dp = ct.POINTER(ct.c_double)
_ip = ct.POINTER(ct.c_int)


class _Master(ct.Structure):
    _fields_ = [("nd", ct.c_int), ("npv", ct.c_int), ("npf", ct.c_int), ("nfe", ct.c_int),
                ("ngv", ct.c_int), ("ngf", ct.c_int), ("shapvt", _dp), ("shapvg", _dp),
                ("shapmv", _dp), ("shapft", _dp), ("shapfg", _dp), ("shapmf", _dp), ("perm", _ip)]


class _App(ct.Structure):
    _fields_ = [("nd", ct.c_int), ("ncu", ct.c_int), ("nc", ct.c_int), ("localsolve", ct.c_int),
                ("fc_q", ct.c_double), ("param", _dp), ("nbnd", ct.c_int), ("bcm", _ip), ("bcs", _dp),
                ("fc_u", ct.c_double), ("tdep", ct.c_int), ("fbou_family", ct.c_int)]


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = HERE / "liboracle.so"
        if not path.exists():
            build()
        _LIB = ct.CDLL(str(path))
    return _LIB


def _f(a):
    return np.asfortranarray(a, dtype=np.float64)


def _p(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _keep(master, app):
    keep = []
    def F(a):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))
        keep.append(a)
        return a.ctypes.data_as(_dp)
    def I(a):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel(order="F"))
        keep.append(a)
        return a.ctypes.data_as(_ip)
    m = _Master(master.nd, master.npv, master.npf, master.nfe, master.ngv, master.ngf,
                F(master.shapvt), F(master.shapvg), F(master.shapmv), F(master.shapft),
                F(master.shapfg), F(master.shapmf), I(master.perm))
    a = _App(app.nd, app.ncu, app.nc, app.localsolve, app.fc_q, F(app.param), len(app.bcm),
             I(app.bcm), F(app.bcs), float(getattr(app, "fc_u", 0.0)), int(getattr(app, "tdep", 0)),
             fbou_family(app))
    return m, a, keep


def hdg_elemental(master, app, dgnodes, bf, UDG, UH, SH, intermediates=False, nthreads=1):
    """kernel/hdg_elemental.m on the CPU: returns AE, FE, DUDG, DUDG_DUH (+ the blocks)."""
    L = lib()
    m, a, keep = _keep(master, app)
    npv, nc, ne = UDG.shape
    ncu, ndf = app.ncu, master.npf * master.nfe
    nd = master.nd
    dg, udg, uh, sh = _f(dgnodes), _f(UDG), _f(UH), _f(SH)
    bfi = np.asfortranarray(bf, dtype=np.int32)
    AE = np.zeros((ncu, ndf, ncu, ndf, ne), order="F")
    FE = np.zeros((ncu, ndf, ne), order="F")
    DUDG = np.zeros((npv, nc, ne), order="F")
    DUDG_DUH = np.zeros((npv, nc, ncu, ndf, ne), order="F")
    st = np.zeros(ne, dtype=np.int32)
    blk = {}
    if intermediates:
        blk = dict(M=np.zeros((npv, npv, ne), order="F"), C=np.zeros((npv, npv, nd, ne), order="F"),
                   E=np.zeros((npv, ndf, nd, ne), order="F"), BD=np.zeros((npv, ncu, npv, nc, ne), order="F"),
                   F=np.zeros((npv, ncu, ncu, ndf, ne), order="F"), GK=np.zeros((ncu, ndf, npv, nc, ne), order="F"),
                   H=np.zeros((ncu, ndf, ncu, ndf, ne), order="F"), Rq=np.zeros((npv, ncu, nd, ne), order="F"),
                   Ru=np.zeros((npv, ncu, ne), order="F"), Rh=np.zeros((ncu, ndf, ne), order="F"))
    g = lambda k: _p(blk.get(k))
    L.orc_hdg_elemental.restype = ct.c_int
    nbad = L.orc_hdg_elemental(ct.byref(m), ct.byref(a), ne, _p(dg), bfi.ctypes.data_as(_ip), _p(udg),
                               _p(uh), _p(sh), _p(AE), _p(FE), _p(DUDG), _p(DUDG_DUH),
                               g("M"), g("C"), g("E"), g("BD"), g("F"), g("GK"), g("H"), g("Rq"),
                               g("Ru"), g("Rh"), st.ctypes.data_as(_ip), int(nthreads))
    if not getattr(app, "getdqdg", 1):       # hdg_elemental.m:20-26: nco = ncu, the u rows only
        ncu = app.ncu
        DUDG, DUDG_DUH = np.asfortranarray(DUDG[:, :ncu]), np.asfortranarray(DUDG_DUH[:, :ncu])
    out = dict(AE=AE, FE=FE, DUDG=DUDG, DUDG_DUH=DUDG_DUH, status=st, nbad=nbad)
    out.update(blk)
    return out


def schur_uq(nd, blocks, nthreads=1):
    """schur_uq2 (kernel/schur_primal.m:52-150) on reference-layout blocks."""
    L = lib()
    M = _f(blocks["M"]); npv, _, ne = M.shape
    ncu = blocks["Ru"].shape[1]; ndf = blocks["E"].shape[1]; nc = ncu * (nd + 1)
    args = [_f(blocks[k]) for k in ("M", "C", "E", "BD", "F", "GK", "H", "Rq", "Ru", "Rh")]
    DUDG = np.zeros((npv, nc, ne), order="F"); DUDG_DUH = np.zeros((npv, nc, ncu, ndf, ne), order="F")
    AE = np.zeros((ncu, ndf, ncu, ndf, ne), order="F"); FE = np.zeros((ncu, ndf, ne), order="F")
    nbad = L.orc_schur_uq(nd, npv, ncu, ndf, ne, *[_p(x) for x in args], _p(DUDG), _p(DUDG_DUH),
                          _p(AE), _p(FE), int(nthreads))
    return dict(DUDG=DUDG, DUDG_DUH=DUDG_DUH, AE=AE, FE=FE, nbad=nbad)


def flux_points(nd, param, udg):
    L = lib(); ng, nc = udg.shape; ncu = nd + 2
    f = np.zeros((ng, ncu, nd), order="F"); fu = np.zeros((ng, ncu, nd, nc), order="F")
    L.orc_flux_points(nd, _p(_f(param)), ng, _p(_f(udg)), _p(f), _p(fu))
    return f, fu


def fbou_family(app):
    """0: application/FM/ns/fbou.m, 1: application/FM/euler/fbou.m (the app's physics folder)."""
    return 1 if getattr(app, "fbou", "ns") == "euler" else 0


def fbou_points(fam, nd, ib, uinf, param, nl, udg, uh):
    """fbou of family fam (0 ns, 1 euler) at ng points: fh[ng,ncu], fh_udg[ng,ncu,nc], fh_uh[ng,ncu,ncu]."""
    L = lib(); ng, nc = udg.shape; ncu = nd + 2
    fh = np.zeros((ng, ncu), order="F"); fhu = np.zeros((ng, ncu, nc), order="F"); fhh = np.zeros((ng, ncu, ncu), order="F")
    rc = L.orc_fbou_points(int(fam), nd, int(ib), _p(_f(uinf)), _p(_f(param)), ng, _p(_f(nl)), _p(_f(udg)), _p(_f(uh)),
                           _p(fh), _p(fhu), _p(fhh))
    if rc:
        raise ValueError(f"boundary type {ib} of family {fam} is not restated")
    return fh, fhu, fhh


def getan_points(nd, param, absolute, nl, uh):
    """Roe matrices of getan.m at ng trace states: An[ng,ncu,ncu], Anm[ng,ncu,ncu,ncu]."""
    L = lib(); ng = uh.shape[0]; ncu = nd + 2
    An = np.zeros((ng, ncu, ncu), order="F"); Anm = np.zeros((ng, ncu, ncu, ncu), order="F")
    L.orc_getan_points(nd, _p(_f(param)), int(absolute), ng, _p(_f(nl)), _p(_f(uh)), _p(An), _p(Anm))
    return An, Anm


def fhat_points(nd, param, nl, udg, uh):
    L = lib(); ng, nc = udg.shape; ncu = nd + 2
    fh = np.zeros((ng, ncu), order="F"); fhu = np.zeros((ng, ncu, nc), order="F"); fhh = np.zeros((ng, ncu, ncu), order="F")
    L.orc_fhat_points(nd, _p(_f(param)), ng, _p(_f(nl)), _p(_f(udg)), _p(_f(uh)), _p(fh), _p(fhu), _p(fhh))
    return fh, fhu, fhh


# ------------------------------------------------------------- compiled reference
def ref_available():
    return (HERE / "_ref" / "schur_uq.so").exists()


def _ref(name):
    if name not in _REF:
        path = HERE / "_ref" / name
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run oracle/build_ref.sh in a tree with the reference")
        _REF[name] = ct.CDLL(str(path))
    return _REF[name]


def ref_mex(soname, inputs, out_shapes):
    """Run a reference mexFunction (oracle/_ref/<soname>) on Fortran-ordered inputs."""
    L = _ref(soname)
    ins = [np.array(x, dtype=np.float64, order="F", copy=True) for x in inputs]   # MEX overwrites inputs
    ptrs = (_dp * len(ins))(*[_p(x) for x in ins])
    ndims = (ct.c_int * len(ins))(*[x.ndim for x in ins])
    dims = [d for x in ins for d in x.shape]
    cd = (ct.c_longlong * len(dims))(*dims)
    outs = [np.zeros(s, order="F") for s in out_shapes]
    optr = (_dp * len(outs))(*[_p(x) for x in outs])
    numel = (ct.c_longlong * len(outs))()
    rc = L.ref_call(len(ins), ptrs, ndims, cd, len(outs), optr, numel)
    if rc != 0:
        raise RuntimeError(f"reference mexFunction failed ({rc})")
    return outs


def ref_mex_call(soname, inputs, out_shapes):
    """A prepared call of a reference mexFunction: returns (run, outs), where run() executes only
    the compiled MEX on private copies of the inputs (each prepared call runs once: the MEX
    overwrites some inputs in place).  For timing the reference's own code alone."""
    L = _ref(soname)
    ins = [np.array(x, dtype=np.float64, order="F", copy=True) for x in inputs]
    ptrs = (_dp * len(ins))(*[_p(x) for x in ins])
    ndims = (ct.c_int * len(ins))(*[x.ndim for x in ins])
    dims = [d for x in ins for d in x.shape]
    cd = (ct.c_longlong * len(dims))(*dims)
    outs = [np.zeros(s, order="F") for s in out_shapes]
    optr = (_dp * len(outs))(*[_p(x) for x in outs])
    numel = (ct.c_longlong * len(outs))()

    def run():
        if L.ref_call(len(ins), ptrs, ndims, cd, len(outs), optr, numel) != 0:
            raise RuntimeError("reference mexFunction failed")
        return ins
    return run, outs


def ref_flux(nd, param, udg, family="ns"):
    """Reference generated flux kernel; family "euler" takes the u-only state (nc = ncu)."""
    L = _ref("libref_ns.so"); ng, nc = udg.shape; ncu = nd + 2
    f = np.zeros((ng, ncu, nd), order="F"); fu = np.zeros((ng, ncu, nd, nc), order="F")
    pg = np.zeros((ng, nd), order="F")
    fn = getattr(L, f"flux_{family}{nd}d")
    fn(_p(f), _p(fu), _p(pg), _p(_f(udg)), _p(_f(param)), ct.c_double(0.0), ng, nc, ncu, nd, nd)
    return f, fu


def ref_fhat(nd, param, nl, udg, uh, family="ns"):
    L = _ref("libref_ns.so"); ng, nc = udg.shape; ncu = nd + 2
    fh = np.zeros((ng, ncu), order="F"); fhu = np.zeros((ng, ncu, nc), order="F"); fhh = np.zeros((ng, ncu, ncu), order="F")
    pg = np.zeros((ng, nd), order="F")
    fn = getattr(L, f"fhat_{family}{nd}d")
    fn(_p(fh), _p(fhu), _p(fhh), _p(pg), _p(_f(udg)), _p(_f(uh)), _p(_f(nl)), _p(_f(param)),
       ct.c_double(0.0), ng, nc, ncu, nd, nd)
    return fh, fhu, fhh


# ------------------------------------------------------------- condensed system (CPU)
_lp = ct.POINTER(ct.c_longlong)


def _i32(a):
    return np.ascontiguousarray(np.asarray(a).ravel(order="F"), dtype=np.int32)


def _i64(a):
    return np.ascontiguousarray(np.asarray(a).ravel(order="F"), dtype=np.int64)


def globalassembly(mesh, AE, FE, npf, ncu):
    """kernel/globalassembly.m: block-CSR Hg[bs,bs,nnzb], Rg[bs,nf]."""
    L = lib()
    ne, nfe = mesh.t2f.shape
    bs = ncu * npf
    nnzb = int(mesh.cbsr_rowpts[-1])
    Hg = np.zeros((bs, bs, nnzb), order="F"); Rg = np.zeros((bs, mesh.nf), order="F")
    t2f, el, rp, ci = _i32(mesh.t2f), _i32(mesh.elcon), _i64(mesh.cbsr_rowpts), _i32(mesh.cbsr_colind)
    L.orc_globalassembly(ne, nfe, npf, ncu, t2f.ctypes.data_as(_ip), el.ctypes.data_as(_ip), mesh.nf,
                         rp.ctypes.data_as(_lp), ci.ctypes.data_as(_ip), _p(_f(AE)), _p(_f(FE)), _p(Hg), _p(Rg))
    return Hg, Rg


def matvec(mesh, Hg, x):
    L = lib(); bs = Hg.shape[0]
    rp, ci = _i64(mesh.cbsr_rowpts), _i32(mesh.cbsr_colind)
    y = np.zeros((bs, mesh.nf), order="F")
    L.orc_matvec(mesh.nf, bs, rp.ctypes.data_as(_lp), ci.ctypes.data_as(_ip), _p(_f(Hg)), _p(_f(x)), _p(y))
    return y


def mdf_ordering(mesh, Hg):
    """kernel/computeMDFordering.m -> (ordered2unordered, unordered2ordered), 0-based."""
    L = lib(); bs = Hg.shape[0]
    rp, ci = _i64(mesh.cbsr_rowpts), _i32(mesh.cbsr_colind)
    o2u = np.zeros(mesh.nf, dtype=np.int32); u2o = np.zeros(mesh.nf, dtype=np.int32)
    L.orc_mdf_ordering(mesh.nf, bs, rp.ctypes.data_as(_lp), ci.ctypes.data_as(_ip), _p(_f(Hg)),
                       o2u.ctypes.data_as(_ip), u2o.ctypes.data_as(_ip))
    return o2u, u2o


def bilu0(mesh, Hg, o2u, u2o):
    """kernel/computeBILU0.m with the given ordering; returns (Mg, status)."""
    L = lib(); bs = Hg.shape[0]
    rp, ci = _i64(mesh.cbsr_rowpts), _i32(mesh.cbsr_colind)
    Mg = np.array(Hg, dtype=np.float64, order="F", copy=True)
    rc = L.orc_bilu0(mesh.nf, bs, rp.ctypes.data_as(_lp), ci.ctypes.data_as(_ip), _i32(o2u).ctypes.data_as(_ip),
                     _i32(u2o).ctypes.data_as(_ip), _p(Mg))
    return Mg, rc


def bilu0_apply(mesh, Mg, x, o2u, u2o):
    L = lib(); bs = Mg.shape[0]
    rp, ci = _i64(mesh.cbsr_rowpts), _i32(mesh.cbsr_colind)
    v = np.zeros((bs, mesh.nf), order="F")
    L.orc_bilu0_apply(mesh.nf, bs, rp.ctypes.data_as(_lp), ci.ctypes.data_as(_ip), _i32(o2u).ctypes.data_as(_ip),
                      _i32(u2o).ctypes.data_as(_ip), _p(_f(Mg)), _p(_f(x)), _p(v))
    return v


def gmres_bilu0(mesh, Mg, Hg, b, x0, o2u, u2o, restart=20, tol=1e-10, maxit=1000):
    """kernel/gmres_bilu0.m -> (x, flag, iter, rev)."""
    L = lib(); bs = Hg.shape[0]
    rp, ci = _i64(mesh.cbsr_rowpts), _i32(mesh.cbsr_colind)
    x = np.array(x0, dtype=np.float64, order="F", copy=True)
    flag = ct.c_int(0); rev = np.zeros(maxit + 1)
    it = L.orc_gmres_bilu0(mesh.nf, bs, rp.ctypes.data_as(_lp), ci.ctypes.data_as(_ip), _i32(o2u).ctypes.data_as(_ip),
                           _i32(u2o).ctypes.data_as(_ip), _p(_f(Mg)), _p(_f(Hg)), _p(_f(b)), _p(x), int(restart),
                           ct.c_double(tol), int(maxit), ct.byref(flag), _p(rev))
    return x, flag.value, it, rev[:it]


def backsub(mesh, DUDG, DUDG_DUH, DUH):
    """hdg_solve.m:119-121 on the CPU."""
    L = lib()
    npv, nc, ne = DUDG.shape
    ncu, ndf = DUDG_DUH.shape[2], DUDG_DUH.shape[3]
    out = np.zeros((npv, nc, ne), order="F")
    L.orc_backsub(ne, npv, nc, ncu, ndf, _i32(mesh.elcon).ctypes.data_as(_ip), _p(_f(DUDG)), _p(_f(DUDG_DUH)),
                  _p(_f(DUH)), _p(out))
    return out


def hdg_solve(P, o2u=None, u2o=None, tol=1e-10, maxiter=16, gmres_tol=1e-10, restart=20, nthreads=1):
    """kernel/hdg_solve.m:104-176 on the CPU (oracle elemental + globalassembly + BILU(0)
    ordered by o2u (MDF when None) + GMRES + back-substitution + damped line search).
    Returns (UDG, UH, residuals, gmres_iters, alphas)."""
    m, a, mesh = P.master, P.app, P.mesh
    npf, ncu = m.npf, a.ncu
    UDG = np.array(P.UDG, order="F", copy=True)
    UH = np.array(P.UH, order="F", copy=True)
    SH = np.array(P.SH, order="F", copy=True)
    SH[:, ncu:, :] = 0.0                         # hdg_solve.m:62-63 (app.wave == 0)

    def assemble(UDG, UH):
        from hdg_b200.app import gather_uh
        r = hdg_elemental(m, a, mesh.dgnodes, mesh.bf, UDG, gather_uh(UH, mesh.elcon), SH, nthreads=nthreads)
        Hg, Rg = globalassembly(mesh, r["AE"], r["FE"], npf, ncu)
        return r, Hg, Rg

    r, Hg, Rg = assemble(UDG, UH)
    F0 = float(np.linalg.norm(Rg))
    res, gits, alphas = [F0], [], []
    F = F0
    rel, it = 1.0, 0
    while rel > tol and it < maxiter:
        if o2u is None:
            oo, uu = mdf_ordering(mesh, Hg)
        else:
            oo, uu = o2u, u2o
        Mg, _ = bilu0(mesh, Hg, oo, uu)
        DUH, flag, gi, _ = gmres_bilu0(mesh, Mg, Hg, Rg, np.zeros_like(Rg), oo, uu, restart, gmres_tol, 1000)
        gits.append(gi)
        DUH = DUH.reshape(ncu, mesh.nsiz, order="F")
        DUDGT = backsub(mesh, r["DUDG"], r["DUDG_DUH"], DUH)
        it += 1
        UDG0, UH0, duh0 = UDG.copy(), UH.copy(), F
        alfa = 1.0
        nco = DUDGT.shape[1]
        while True:
            UDG = UDG0.copy()
            UDG[:, :nco, :] += alfa * DUDGT                      # hdg_solve.m:145-146
            UH = UH0 + alfa * DUH
            if nco < a.nc:                                        # getdqdg = 0: hdg_solve.m:148-151
                from hdg_b200.app import gather_uh
                UDG[:, ncu:, :] = getq(m, a, mesh.dgnodes, mesh.bf, UDG, gather_uh(UH, mesh.elcon), SH, a.fc_q)
            r, Hg, Rg = assemble(UDG, UH)
            F = float(np.linalg.norm(Rg))
            if F > duh0:
                alfa /= 2
                if alfa < 1e-2:
                    break
            else:
                break
        alphas.append(alfa)
        res.append(F)
        rel = F / F0
    return UDG, UH, res, gits, alphas


def dense_block_system(mesh, AE, FE, npf, ncu):
    """mkf2f.m + mkDenseBlockSystem.m (from the elemental arrays): (f2f, K, F)."""
    L = lib()
    ne, nfe = mesh.t2f.shape
    nf = mesh.nf
    nbf = 2 * nfe - 1
    ncf = ncu * npf
    fel = np.ascontiguousarray(np.asarray(mesh.f)[:, -2:], dtype=np.int32).ravel()
    f2f = np.zeros((nbf, nf), dtype=np.int32, order="F")
    K = np.zeros((ncf, ncf * (nbf - 1), nf), order="F")
    F = np.zeros((ncf, nf), order="F")
    t2f, el = _i32(np.abs(mesh.t2f)), _i32(mesh.elcon)
    L.orc_dense_block_system.restype = ct.c_int
    nbad = L.orc_dense_block_system(ne, nfe, npf, ncu, nf, fel.ctypes.data_as(_ip), t2f.ctypes.data_as(_ip),
                                    el.ctypes.data_as(_ip), _p(_f(AE)), _p(_f(FE)), f2f.ctypes.data_as(_ip),
                                    _p(K), _p(F))
    if nbad:
        raise RuntimeError(f"{nbad} singular diagonal blocks")
    return f2f, K, F


def dense_matvec(K, f2f, x):
    L = lib()
    nb, nf = x.shape
    nbf = f2f.shape[0]
    y = np.zeros((nb, nf), order="F")
    f2 = _i32(f2f)
    L.orc_dense_matvec(nb, nf, nbf, _p(_f(K)), f2.ctypes.data_as(_ip), _p(_f(x)), _p(y))
    return y


def gmres_dense(K, F, f2f, x0=None, restart=20, tol=1e-6, maxit=None):
    """kernel/gmres.m: returns (x, flag, iterations, relative residual history)."""
    L = lib()
    nb, nf = F.shape
    nbf = f2f.shape[0]
    maxit = nb * nf if maxit is None else maxit
    x = np.zeros((nb, nf), order="F") if x0 is None else np.array(x0, dtype=np.float64, order="F")
    rev = np.zeros(maxit)
    flag = ct.c_int(0)
    f2 = _i32(f2f)
    L.orc_gmres_dense.restype = ct.c_int
    it = L.orc_gmres_dense(nb, nf, nbf, _p(_f(K)), f2.ctypes.data_as(_ip), _p(_f(F)), _p(x), int(restart),
                           ct.c_double(tol), int(maxit), ct.byref(flag), _p(rev))
    return x, flag.value, it, rev[:it]


def dirkcoeff(q, p):
    """kernel/hdg_solve_dirk.m (dirkcoeff): Butcher tableau of the (stages q, order p) DIRK
    scheme as (d = inv(a), c = b inv(a), t)."""
    s2, s3 = np.sqrt(2.0), np.sqrt(3.0)
    tab = {
        (1, 1): ([[1.0]], [1.0], [1.0]),
        (1, 2): ([[0.5]], [1.0], [0.5]),
        (2, 2): ([[1 - 0.5 * s2, 0], [0.5 * s2, 1 - 0.5 * s2]], [0.5 * s2, 1 - 0.5 * s2], [1 - 0.5 * s2, 1]),
        (2, 3): ([[0.5 + 0.5 / s3, 0], [-1 / s3, 0.5 + 0.5 / s3]], [0.5, 0.5], [0.5 + 0.5 / s3, 0.5 - 0.5 / s3]),
    }
    if (q, p) == (3, 3):
        a1 = 0.4358665215
        t1 = (1 + a1) / 2
        b1 = -(6 * a1 ** 2 - 16 * a1 + 1) / 4
        b2 = (6 * a1 ** 2 - 20 * a1 + 5) / 4
        tab[(3, 3)] = ([[a1, 0, 0], [t1 - a1, a1, 0], [b1, b2, a1]], [b1, b2, a1], [a1, t1, 1])
    if (q, p) == (3, 4):
        a1 = 2 * np.cos(np.pi / 18) / s3
        tab[(3, 4)] = ([[0.5 * (1 + a1), 0, 0], [-0.5 * a1, 0.5 * (1 + a1), 0], [1 + a1, -(1 + 2 * a1), 0.5 * (1 + a1)]],
                       [1 / (6 * a1 ** 2), 1 - 1 / (3 * a1 ** 2), 1 / (6 * a1 ** 2)],
                       [0.5 * (1 + a1), 0.5, 0.5 * (1 - a1)])
    a, b, t = (np.array(x, dtype=np.float64) for x in tab[(q, p)])
    d = np.linalg.inv(a)
    return d, b @ d, t


def hdg_solve_dirk(P, time, dt, nstage, torder, tol=1e-10, maxiter=16, gmres_tol=1e-10, nthreads=1):
    """kernel/hdg_solve_dirk.m:1-80 on the CPU, one step from (P.UDG, P.UH): each stage forms
    its source SDG, resets the q part of UDG with getq (components ncu+1:nc), and is the oracle
    hdg_solve of the time-dependent residual (app.tdep = 1, fc_u = d(s,s), fc_q = 1).
    Returns (Un, Hn)."""
    import copy
    from types import SimpleNamespace
    d, c, t = dirkcoeff(nstage, torder)
    d = d / dt
    UDG = np.asarray(P.UDG, dtype=np.float64)
    UH = np.asarray(P.UH, dtype=np.float64)
    Un = (1 - c.sum()) * UDG
    Hn = (1 - c.sum()) * UH
    UDGn, SDG = [], None
    for s in range(nstage):
        if s == 0:
            SDG = d[0, 0] * UDG
        elif s == 1:
            SDG = (d[1, 0] + d[1, 1]) * UDG - d[1, 0] * UDGn[0]
        else:
            SDG = ((d[2, 0] + d[2, 1] + d[2, 2]) * UDG - (d[2, 0] / d[1, 0]) * ((d[1, 0] + d[1, 1]) * UDG - SDG)
                   - d[2, 1] * UDGn[1])
        app = copy.copy(P.app)
        app.fc_u, app.fc_q, app.tdep = float(d[s, s]), 1.0, 1
        from hdg_b200.app import gather_uh
        UDG = np.array(UDG, copy=True)
        UDG[:, app.ncu:, :] = getq(P.master, app, P.mesh.dgnodes, P.mesh.bf, UDG, gather_uh(UH, P.mesh.elcon),
                                   None, app.fc_q)
        Q = SimpleNamespace(master=P.master, app=app, mesh=P.mesh, UDG=UDG, UH=UH, SH=SDG)
        Us, Hs, _, _, _ = hdg_solve(Q, tol=tol, maxiter=maxiter, gmres_tol=gmres_tol, nthreads=nthreads)
        UDGn.append(Us)
        Un = Un + c[s] * Us
        Hn = Hn + c[s] * Hs
    return Un, Hn


def schur_uq_adjoint(M, C, E, BD, F, GK, H, Rq, Ru, Rh):
    """kernel/schur_uq_adjoint.c (localsolveuq :43-298) restated with numpy, per element:
    SDt = D^T + sum_n C_n^T Mi B_n^T, [du, dlu] = SDt \\ [Ru + sum_n C_n^T Mi Rq_n,
    -(K^T + sum_n C_n^T Mi G_n^T)], dq_n = Mi (Rq_n - B_n^T du), dlq_n = -Mi (B_n^T dlu + G_n^T),
    FE = Rh - F^T du - sum_n E_n^T dq_n, AE = H^T + F^T dlu + sum_n E_n^T dlq_n
    (Mi, C_n^T, E_n^T act on the node index of every component)."""
    npv, ncu, _, nc, ne = BD.shape
    nd = C.shape[2]; ndf = E.shape[1]; nu, nh = npv * ncu, ncu * ndf
    DUDG = np.zeros((npv, nc, ne), order="F"); DD = np.zeros((npv, nc, ncu, ndf, ne), order="F")
    AE = np.zeros((ncu, ndf, ncu, ndf, ne), order="F"); FE = np.zeros((ncu, ndf, ne), order="F")
    mat = lambda a, r, c: a.reshape((r, c), order="F")
    for e in range(ne):
        Mi = np.linalg.inv(M[:, :, e])
        node = lambda A, X: np.einsum("st,tb...->sb...", A, X)      # act on the node index
        D = mat(BD[:, :, :, :ncu, e], nu, nu)
        K = mat(GK[:, :, :, :ncu, e], nh, nu)
        SDt = D.T.copy()
        R0 = Ru[:, :, e].copy()
        KT = K.T.reshape((npv, ncu, nh), order="F").copy()
        Bn = [mat(BD[:, :, :, ncu + ncu * n:2 * ncu + ncu * n, e], nu, nu) for n in range(nd)]
        Gn = [mat(GK[:, :, :, ncu + ncu * n:2 * ncu + ncu * n, e], nh, nu) for n in range(nd)]
        for n in range(nd):
            W = C[:, :, n, e].T @ Mi
            SDt += mat(node(W, Bn[n].T.reshape((npv, ncu, nu), order="F")), nu, nu)
            R0 += W @ Rq[:, :, n, e]
            KT += node(W, Gn[n].T.reshape((npv, ncu, nh), order="F"))
        X = np.linalg.solve(SDt, np.column_stack([R0.ravel(order="F"), -mat(KT, nu, nh)]))
        du, dlu = X[:, 0], X[:, 1:]
        dq = [node(Mi, Rq[:, :, n, e] - (Bn[n].T @ du).reshape((npv, ncu), order="F")) for n in range(nd)]
        dlq = [-node(Mi, (Bn[n].T @ dlu + Gn[n].T).reshape((npv, ncu, nh), order="F")) for n in range(nd)]
        DUDG[:, :ncu, e] = du.reshape((npv, ncu), order="F")
        DD[:, :ncu, :, :, e] = dlu.reshape((npv, ncu, ncu, ndf), order="F")
        for n in range(nd):
            DUDG[:, ncu + ncu * n:2 * ncu + ncu * n, e] = dq[n]
            DD[:, ncu + ncu * n:2 * ncu + ncu * n, :, :, e] = dlq[n].reshape((npv, ncu, ncu, ndf), order="F")
        Ft = mat(F[:, :, :, :, e], nu, nh).T
        fe = Rh[:, :, e].ravel(order="F") - Ft @ du
        ae = mat(H[:, :, :, :, e], nh, nh).T + Ft @ dlu
        for n in range(nd):
            En = E[:, :, n, e]                                          # [npv, ndf]
            fe -= (En.T @ dq[n]).T.ravel(order="F")                     # (a, f) <- sum_s E(s,f) dq(s,a)
            ae += np.einsum("sf,sak->afk", En, dlq[n]).reshape((nh, nh), order="F")
        FE[:, :, e] = fe.reshape((ncu, ndf), order="F")
        AE[:, :, :, :, e] = ae.reshape((ncu, ndf, ncu, ndf), order="F")
    return DUDG, DD, AE, FE


def schur_u_adjoint(BD, F, GK, H, Ru, Rh):
    """kernel/schur_u_adjoint.c (localsolve :43-143) restated with numpy: [du, dlu] = D^T \\
    [Ru, -K^T], FE = Rh - F^T du, AE = H^T + F^T dlu; du and dlu (column-major) fill the start of
    each element's DUDG / DUDG_DUH slab, the rest zero, as that MEX writes them."""
    npv, ncu, _, nc, ne = BD.shape
    ndf = H.shape[1]; nu, nh = npv * ncu, ncu * ndf
    DUDG = np.zeros((npv * nc, ne)); DD = np.zeros((npv * nc * nh, ne))
    AE = np.zeros((nh * nh, ne)); FE = np.zeros((nh, ne))
    for e in range(ne):
        D = BD[:, :, :, :ncu, e].reshape((nu, nu), order="F")
        K = GK[:, :, :, :ncu, e].reshape((nh, nu), order="F")
        X = np.linalg.solve(D.T, np.column_stack([Ru[:, :, e].ravel(order="F"), -K.T]))
        Ft = F[:, :, :, :, e].reshape((nu, nh), order="F").T
        DUDG[:nu, e] = X[:, 0]
        DD[:nu * nh, e] = X[:, 1:].ravel(order="F")
        FE[:, e] = Rh[:, :, e].ravel(order="F") - Ft @ X[:, 0]
        AE[:, e] = (H[:, :, :, :, e].reshape((nh, nh), order="F").T + Ft @ X[:, 1:]).ravel(order="F")
    return (DUDG.reshape((npv, nc, ne), order="F"), DD.reshape((npv, nc, ncu, ndf, ne), order="F"),
            AE.reshape((ncu, ndf, ncu, ndf, ne), order="F"), FE.reshape((ncu, ndf, ne), order="F"))


def getq(master, app, dgnodes, bf, UDG, UHe, SH=None, fc_q=1.0):
    """kernel/getq.m on the CPU: QDG[npv, ncu*nd, ne] = inv(fc_q Mu) (C u - E uh) + SH_q/fc_q, with
    Mu, C, E the oracle's volint/faceint blocks (getq.m's local volgeom negates both the adjugate
    and the face normal, so its Mi (E uh - C u) is this same expression)."""
    import copy
    a = copy.copy(app)
    a.fc_q = float(fc_q)
    a.tdep = 0
    ne = UDG.shape[-1]
    ncu, nd, npv = a.ncu, master.nd, master.npv
    zero = np.zeros_like(UDG)
    blk = hdg_elemental(master, a, dgnodes, bf, UDG, UHe, zero, intermediates=True)
    Q = np.zeros((npv, ncu * nd, ne), order="F")
    for e in range(ne):
        Mi = np.linalg.inv(blk["M"][:, :, e])
        for d in range(nd):
            rhs = blk["C"][:, :, d, e] @ UDG[:, :ncu, e] - blk["E"][:, :, d, e] @ UHe[:, :, e].T
            Q[:, ncu * d:ncu * (d + 1), e] = Mi @ rhs
    if SH is not None:
        Q = Q + np.asarray(SH)[:, ncu:, :] / fc_q
    return Q


def residual(master, app, dgnodes, bf, UDG, UHe, SH=None):
    """kernel/cuda_residual.m on the CPU: q = getq(u, uh, SH, fc_q), then the oracle's element u
    residual Ru (volint + faceint) at that q."""
    ncu = app.ncu
    U = np.array(UDG, dtype=np.float64, copy=True)
    U[:, ncu:, :] = getq(master, app, dgnodes, bf, U, UHe, SH, app.fc_q)
    sh = np.zeros_like(U) if SH is None else SH
    return hdg_elemental(master, app, dgnodes, bf, U, UHe, sh, intermediates=True)["Ru"]
