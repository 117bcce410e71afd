"""Host-side mirror of the reference's elemental call surface, on the GPU through libhdgx.

``hdg_elemental(master, app, dgnodes, bf, UDG, UH, SH)`` has the argument meaning of
``kernel/hdg_elemental.m:1`` and returns ``AE, FE, DUDG, DUDG_DUH`` in the same layouts.
``schur_uq`` / ``schur_u`` mirror the MEX files ``kernel/schur_uq.c`` / ``kernel/schur_u.c``.

Array convention: numpy arrays are indexed like MATLAB (``A[i, j, k]`` is ``A(i+1,j+1,k+1)``)
and may have any memory order; device arrays are ``DArray`` objects: a flat CUDA tensor in
column-major order plus the MATLAB shape.  Host inputs are copied to the device, results
come back as ``DArray`` (``.numpy()`` gives the MATLAB-indexed host array).
"""
from __future__ import annotations

import ctypes as ct
import math
from dataclasses import dataclass

import numpy as np
import torch

from ._lib import HDGX_MAX_BND, HdgxApp, HdgxError, HdgxMaster, check, lib


def _require_cuda():
    if not torch.cuda.is_available():
        raise HdgxError("hdg_b200 compute entry points need a CUDA device (no CPU fallback)")


@dataclass
class DArray:
    """A column-major device array with a MATLAB shape."""
    t: torch.Tensor       # flat, contiguous
    shape: tuple

    @staticmethod
    def empty(shape, dtype=torch.float64, device="cuda"):
        return DArray(torch.empty(int(np.prod(shape)), dtype=dtype, device=device), tuple(int(s) for s in shape))

    @staticmethod
    def zeros(shape, dtype=torch.float64, device="cuda"):
        return DArray(torch.zeros(int(np.prod(shape)), dtype=dtype, device=device), tuple(int(s) for s in shape))

    @staticmethod
    def from_numpy(a, dtype=torch.float64, device="cuda", pin=False):
        a = np.asarray(a)
        flat = np.ascontiguousarray(a.ravel(order="F"))
        t = torch.from_numpy(flat).to(dtype)
        if pin:
            t = t.pin_memory()
        return DArray(t.to(device, non_blocking=pin), tuple(a.shape))

    def numpy(self):
        return self.t.detach().cpu().numpy().reshape(self.shape, order="F")

    def view(self):
        """MATLAB-indexed (non-contiguous) view of the device data."""
        return self.t.view(tuple(reversed(self.shape))).permute(*reversed(range(len(self.shape))))

    @property
    def ptr(self):
        return self.t.data_ptr()


def as_darray(x, dtype=torch.float64):
    if isinstance(x, DArray):
        if x.t.dtype != dtype:
            raise TypeError(f"expected {dtype}, got {x.t.dtype}")
        return x
    return DArray.from_numpy(x, dtype=dtype)


class DeviceMaster:
    """Master element tables resident on the device (``hdgx_master``)."""

    def __init__(self, master):
        _require_cuda()
        self.master = master
        self.nd, self.porder = master.nd, master.porder
        self.npv, self.npf, self.nfe = master.npv, master.npf, master.nfe
        self.ngv, self.ngf = master.ngv, master.ngf
        self.arrays = {k: DArray.from_numpy(getattr(master, k))
                       for k in ("shapvt", "shapvg", "shapmv", "shapft", "shapfg", "shapmf")}
        self.arrays["perm"] = DArray.from_numpy(master.perm, dtype=torch.int32)
        a = self.arrays
        self.c = HdgxMaster(self.nd, self.porder, self.npv, self.npf, self.nfe, self.ngv, self.ngf,
                            a["shapvt"].ptr, a["shapvg"].ptr, a["shapmv"].ptr, a["shapft"].ptr,
                            a["shapfg"].ptr, a["shapmf"].ptr, a["perm"].ptr)


def app_struct(app):
    nb = len(app.bcm)
    if nb > HDGX_MAX_BND:
        raise HdgxError(f"at most {HDGX_MAX_BND} boundary indices are supported")
    s = HdgxApp()
    s.nd, s.ncu, s.nc = app.nd, app.ncu, app.nc
    s.localsolve, s.getdqdg = app.localsolve, app.getdqdg
    s.fc_q, s.fc_u, s.tdep = app.fc_q, app.fc_u, app.tdep
    for i, v in enumerate(np.asarray(app.param, dtype=np.float64)[:8]):
        s.param[i] = float(v)
    s.nbnd = nb
    s.fbou = 1 if getattr(app, "fbou", "ns") == "euler" else 0
    for i in range(nb):
        s.bcm[i] = int(app.bcm[i])
        for a in range(app.ncu):
            s.bcs[i * 5 + a] = float(app.bcs[i][a])
    return s


def _stream_ptr(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return ct.c_void_p(stream.cuda_stream)


class ElementalOutputs:
    def __init__(self, AE, FE, DUDG, DUDG_DUH, status):
        self.AE, self.FE, self.DUDG, self.DUDG_DUH, self.status = AE, FE, DUDG, DUDG_DUH, status

    def __iter__(self):
        return iter((self.AE, self.FE, self.DUDG, self.DUDG_DUH))


def stored_components(app):
    """Components of DUDG / DUDG_DUH: nc, or ncu when app.getdqdg = 0 (hdg_elemental.m:20-26)."""
    return app.nc if getattr(app, "getdqdg", 1) else app.ncu


def alloc_elemental_outputs(master, app, ne):
    npv, ncu, nco = master.npv, app.ncu, stored_components(app)
    ndf = master.npf * master.nfe
    return ElementalOutputs(DArray.empty((ncu, ndf, ncu, ndf, ne)), DArray.empty((ncu, ndf, ne)),
                            DArray.empty((npv, nco, ne)), DArray.empty((npv, nco, ncu, ndf, ne)),
                            DArray.zeros((ne,), dtype=torch.int32))


def hdg_elemental(master, app, dgnodes, bf, UDG, UH, SH, out=None, stream=None, dmaster=None, mixed=False):
    """kernel/hdg_elemental.m: [AE, FE, DUDG, DUDG_DUH] for every element, on the GPU.

    ``mixed=True`` selects the mixed-precision kernel (FP32 local elimination of the Jacobian
    columns, FP64-refined residual solve): FE and DUDG stay FP64-accurate, AE and DUDG_DUH
    carry FP32-level error.

    ``UH`` is the element-gathered trace ``[ncu, npf*nfe, ne]`` (hdg_assemble.m:34).
    Returns an ``ElementalOutputs`` (iterable as AE, FE, DUDG, DUDG_DUH) of ``DArray``s;
    ``status[e]`` is 0, or 1/2 for a singular mass / local matrix, 3 for an unsupported
    boundary type.
    """
    _require_cuda()
    L = lib()
    dm = dmaster if dmaster is not None else DeviceMaster(master)
    ne = int(np.asarray(UDG.shape)[-1]) if not isinstance(UDG, DArray) else UDG.shape[-1]
    dg, udg, uh, sh = (as_darray(x) for x in (dgnodes, UDG, UH, SH))
    bfd = as_darray(bf, dtype=torch.int32)
    o = out if out is not None else alloc_elemental_outputs(master, app, ne)
    a = app_struct(app)
    fn = L.hdgx_elemental_mixed if mixed else L.hdgx_elemental
    rc = fn(ct.byref(dm.c), ct.byref(a), ne, dg.ptr, bfd.ptr, udg.ptr, uh.ptr, sh.ptr,
            o.AE.ptr, o.FE.ptr, o.DUDG.ptr, o.DUDG_DUH.ptr, o.status.ptr, _stream_ptr(stream))
    check(rc, "hdgx_elemental_mixed" if mixed else "hdgx_elemental")
    return o


def getq(master, app, dgnodes, bf, UDG, UH, SH=None, fc_q=None, stream=None, dmaster=None):
    """kernel/getq.m: QDG[npv, ncu*nd, ne], the q that zeroes the local q equation for the
    given u and element-gathered trace UH (``SH`` None: no source, as getq(...,[],fc_q));
    ``fc_q`` defaults to ``app.fc_q``.  Returns (QDG, status) as DArrays."""
    import copy
    _require_cuda()
    L = lib()
    dm = dmaster if dmaster is not None else DeviceMaster(master)
    if fc_q is not None:
        app = copy.copy(app)
        app.fc_q = float(fc_q)
    dg, udg, uh = (as_darray(x) for x in (dgnodes, UDG, UH))
    sh = as_darray(SH) if SH is not None else None
    bfd = as_darray(bf, dtype=torch.int32)
    ne = udg.shape[-1]
    Q = DArray.empty((master.npv, app.ncu * master.nd, ne))
    st = DArray.zeros((ne,), dtype=torch.int32)
    a = app_struct(app)
    rc = L.hdgx_getq(ct.byref(dm.c), ct.byref(a), ne, dg.ptr, bfd.ptr, udg.ptr, uh.ptr, sh.ptr if sh else None,
                     Q.ptr, st.ptr, _stream_ptr(stream))
    check(rc, "hdgx_getq")
    return Q, st


def residual(master, app, dgnodes, bf, UDG, UH, SH=None, stream=None, dmaster=None):
    """kernel/cuda_residual.m: the element u residual Ru[npv, ncu, ne] at q = getq(u, uh), with
    no Jacobian and no local solve (explicit / residual-only evaluation).  Returns (Ru, status)."""
    _require_cuda()
    L = lib()
    dm = dmaster if dmaster is not None else DeviceMaster(master)
    dg, udg, uh = (as_darray(x) for x in (dgnodes, UDG, UH))
    sh = as_darray(SH) if SH is not None else None
    bfd = as_darray(bf, dtype=torch.int32)
    ne = udg.shape[-1]
    Ru = DArray.empty((master.npv, app.ncu, ne))
    st = DArray.zeros((ne,), dtype=torch.int32)
    a = app_struct(app)
    rc = L.hdgx_residual(ct.byref(dm.c), ct.byref(a), ne, dg.ptr, bfd.ptr, udg.ptr, uh.ptr, sh.ptr if sh else None,
                         Ru.ptr, st.ptr, _stream_ptr(stream))
    check(rc, "hdgx_residual")
    return Ru, st


def as_host_darray(x, dtype=torch.float64):
    """A column-major page-locked host DArray of ``x`` (a numpy array, or a host DArray kept as is)."""
    if isinstance(x, DArray):
        if x.t.is_cuda:
            raise HdgxError("expected a host array, got device memory")
        if x.t.dtype != dtype:
            raise TypeError(f"expected {dtype}, got {x.t.dtype}")
        return x
    a = np.asarray(x)
    t = torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).to(dtype).pin_memory()
    return DArray(t, tuple(a.shape))


def alloc_host_outputs(master, app, ne):
    """Page-locked host outputs of hdg_elemental_host."""
    npv, ncu, nc = master.npv, app.ncu, stored_components(app)
    ndf = master.npf * master.nfe

    def pinned(shape, dtype=torch.float64):
        return DArray(torch.empty(int(np.prod(shape)), dtype=dtype, pin_memory=True), tuple(int(x) for x in shape))
    return ElementalOutputs(pinned((ncu, ndf, ncu, ndf, ne)), pinned((ncu, ndf, ne)), pinned((npv, nc, ne)),
                            pinned((npv, nc, ncu, ndf, ne)), pinned((ne,), torch.int32))


def hdg_elemental_host(master, app, dgnodes, bf, UDG, UH, SH, out=None, stream=None, dmaster=None, mixed=False,
                       chunk=0):
    """kernel/hdg_elemental.m on HOST arrays, as the reference is called: the per-element inputs
    and outputs stay in page-locked host memory and the library streams them through the GPU in
    chunks of ``chunk`` elements (0: its default), overlapping the uploads, the kernel and the
    downloads.  Arguments as ``hdg_elemental``; returns ``ElementalOutputs`` of host ``DArray``s,
    bitwise equal to the device-array call's.  Returns when the outputs are in host memory."""
    _require_cuda()
    L = lib()
    dm = dmaster if dmaster is not None else DeviceMaster(master)
    dg, udg, uh, sh = (as_host_darray(x) for x in (dgnodes, UDG, UH, SH))
    bfh = as_host_darray(bf, dtype=torch.int32)
    ne = udg.shape[-1]
    o = out if out is not None else alloc_host_outputs(master, app, ne)
    a = app_struct(app)
    rc = L.hdgx_elemental_host(ct.byref(dm.c), ct.byref(a), ne, dg.ptr, bfh.ptr, udg.ptr, uh.ptr, sh.ptr,
                               o.AE.ptr, o.FE.ptr, o.DUDG.ptr, o.DUDG_DUH.ptr, o.status.ptr, int(bool(mixed)),
                               int(chunk), _stream_ptr(stream))
    check(rc, "hdgx_elemental_host")
    return o


def schur_uq(M, C, E, BD, F, GK, H, Rq, Ru, Rh, stream=None):
    """kernel/schur_uq.c: [DUDG, DUDG_DUH, AE, FE] from the reference's elemental blocks."""
    _require_cuda()
    L = lib()
    arrs = [as_darray(x) for x in (M, C, E, BD, F, GK, H, Rq, Ru, Rh)]
    npv, ne = arrs[0].shape[0], arrs[0].shape[-1]
    ndf, nd = arrs[2].shape[1], arrs[2].shape[2]
    ncu, nc = arrs[3].shape[1], arrs[3].shape[3]
    DUDG = DArray.empty((npv, nc, ne)); DD = DArray.empty((npv, nc, ncu, ndf, ne))
    AE = DArray.empty((ncu, ndf, ncu, ndf, ne)); FE = DArray.empty((ncu, ndf, ne))
    st = DArray.zeros((ne,), dtype=torch.int32)
    rc = L.hdgx_schur_uq(nd, npv, ncu, ndf, ne, *[x.ptr for x in arrs], DUDG.ptr, DD.ptr, AE.ptr, FE.ptr,
                         st.ptr, _stream_ptr(stream))
    check(rc, "hdgx_schur_uq")
    return DUDG, DD, AE, FE, st


def schur_u(BD, F, GK, H, Ru, Rh, stream=None):
    """kernel/schur_u.c: u-only local Schur complement."""
    _require_cuda()
    L = lib()
    arrs = [as_darray(x) for x in (BD, F, GK, H, Ru, Rh)]
    npv, ncu, nc, ne = arrs[0].shape[0], arrs[0].shape[1], arrs[0].shape[3], arrs[0].shape[-1]
    ndf = arrs[1].shape[3]
    DUDG = DArray.empty((npv, nc, ne)); DD = DArray.empty((npv, nc, ncu, ndf, ne))
    AE = DArray.empty((ncu, ndf, ncu, ndf, ne)); FE = DArray.empty((ncu, ndf, ne))
    st = DArray.zeros((ne,), dtype=torch.int32)
    rc = L.hdgx_schur_u(npv, ncu, nc, ndf, ne, *[x.ptr for x in arrs], DUDG.ptr, DD.ptr, AE.ptr, FE.ptr,
                        st.ptr, _stream_ptr(stream))
    check(rc, "hdgx_schur_u")
    return DUDG, DD, AE, FE, st


def schur_uq_adjoint(M, C, E, BD, F, GK, H, Rq, Ru, Rh, stream=None):
    """kernel/schur_uq_adjoint.c: the transposed (adjoint) local Schur complement,
    [DUDG, DUDG_DUH, AE, FE] from the same blocks as ``schur_uq``."""
    _require_cuda()
    L = lib()
    arrs = [as_darray(x) for x in (M, C, E, BD, F, GK, H, Rq, Ru, Rh)]
    npv, ne = arrs[0].shape[0], arrs[0].shape[-1]
    ndf, nd = arrs[2].shape[1], arrs[2].shape[2]
    ncu, nc = arrs[3].shape[1], arrs[3].shape[3]
    DUDG = DArray.empty((npv, nc, ne)); DD = DArray.empty((npv, nc, ncu, ndf, ne))
    AE = DArray.empty((ncu, ndf, ncu, ndf, ne)); FE = DArray.empty((ncu, ndf, ne))
    st = DArray.zeros((ne,), dtype=torch.int32)
    rc = L.hdgx_schur_uq_adjoint(nd, npv, ncu, ndf, ne, *[x.ptr for x in arrs], DUDG.ptr, DD.ptr, AE.ptr, FE.ptr,
                                 st.ptr, _stream_ptr(stream))
    check(rc, "hdgx_schur_uq_adjoint")
    return DUDG, DD, AE, FE, st


def schur_u_adjoint(BD, F, GK, H, Ru, Rh, stream=None):
    """kernel/schur_u_adjoint.c: the transposed u-only local Schur complement (du and dlu fill
    the start of each element's DUDG / DUDG_DUH slab, the rest is zero, as that MEX writes)."""
    _require_cuda()
    L = lib()
    arrs = [as_darray(x) for x in (BD, F, GK, H, Ru, Rh)]
    npv, ncu, nc, ne = arrs[0].shape[0], arrs[0].shape[1], arrs[0].shape[3], arrs[0].shape[-1]
    ndf = arrs[1].shape[3]
    DUDG = DArray.empty((npv, nc, ne)); DD = DArray.empty((npv, nc, ncu, ndf, ne))
    AE = DArray.empty((ncu, ndf, ncu, ndf, ne)); FE = DArray.empty((ncu, ndf, ne))
    st = DArray.zeros((ne,), dtype=torch.int32)
    rc = L.hdgx_schur_u_adjoint(npv, ncu, nc, ndf, ne, *[x.ptr for x in arrs], DUDG.ptr, DD.ptr, AE.ptr, FE.ptr,
                                st.ptr, _stream_ptr(stream))
    check(rc, "hdgx_schur_u_adjoint")
    return DUDG, DD, AE, FE, st
