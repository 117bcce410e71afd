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
                ("fc_q", ct.c_double), ("param", _dp), ("nbnd", ct.c_int), ("bcm", _ip), ("bcs", _dp)]


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
             I(app.bcm), F(app.bcs))
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
