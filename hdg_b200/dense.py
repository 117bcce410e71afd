"""The reference's dense face-block solver path (``app.denseblock = 1`` in kernel/hdg_solve.m:72-74,
88-92, 110-116) on the GPU through libhdgx.

``arraymul(A, B)``           kernel/arraymul.c            batched GEMM / GEMV
``DenseBlockSystem``         kernel/mkDenseBlockSystem.m  inv(D_i)-scaled face blocks K, F
``DenseBlockSystem.gmres``   kernel/gmres.m               GMRES on x + K gather(x, f2f)

The block rows are taken from the assembled block-CSR system (``TraceSystem``), which holds the
same face blocks as mkDenseBlockSystem.m reads from AE / FE; ``f2f`` is mesh/mkmesh/mkf2f.m's
face-to-face table.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

from ._lib import HdgxError, check, lib
from .elemental import DArray, _require_cuda, _stream_ptr, as_darray
from .mesh import mkf2f


def arraymul(A, B, stream=None):
    """kernel/arraymul.c: ``C(:,:,i) = A(:,:,i) * B(:,:,i)``; when B is 2-D with as many
    columns as A has pages, ``C(:,i) = A(:,:,i) * B(:,i)``.  A 2-D A is one page."""
    _require_cuda()
    dA, dB = as_darray(A), as_darray(B)
    sa, sb = dA.shape, dB.shape
    rowsA, colsA = sa[0], (sa[1] if len(sa) > 1 else 1)
    ndim3 = sa[2] if len(sa) == 3 else 1
    rowsB, colsB = sb[0], (sb[1] if len(sb) > 1 else 1)
    ndimB = max(2, len(sb))
    if colsA != rowsB:
        raise HdgxError("Number of columns of A must be equal to numbers of rows B.")
    if ndimB == 2 and colsB == ndim3:
        C = DArray.empty((rowsA, ndim3))
    else:
        if int(np.prod(sb)) != rowsB * colsB * ndim3:
            raise HdgxError("B must hold one rowsB x colsB matrix per page of A")
        C = DArray.empty((rowsA, colsB, ndim3))
    check(lib().hdgx_arraymul(rowsA, colsA, ndim3, rowsB, colsB, ndimB, dA.ptr, dB.ptr, C.ptr, _stream_ptr(stream)),
          "hdgx_arraymul")
    return C


class DenseBlockSystem:
    """K[bs, bs*(nbf-1), nf] and F[bs, nf] of mkDenseBlockSystem.m for a trace system."""

    def __init__(self, ts, mesh):
        _require_cuda()
        self.ts = ts
        self.nf, self.bs = ts.nf, ts.bs
        f2f = mkf2f(mesh.f, mesh.t2f)
        self.nbf = f2f.shape[0]
        self.f2f_h = f2f
        self.f2f = DArray.from_numpy(f2f, dtype=torch.int32)
        self.K = DArray.empty((self.bs, self.bs * (self.nbf - 1), self.nf))
        self.F = DArray.empty((self.bs, self.nf))
        self.status = DArray.zeros((self.nf,), dtype=torch.int32)
        self._ws = {}

    def build(self, Hg, Rg, stream=None):
        """K = inv(D_i) H_i,f2f and F = inv(D_i) R_i for every face i."""
        rc = lib().hdgx_dense_block_system(ct.byref(self.ts.bsr), Hg.ptr, Rg.ptr, self.nbf, self.f2f.ptr, self.K.ptr,
                                           self.F.ptr, self.status.ptr, _stream_ptr(stream))
        check(rc, "hdgx_dense_block_system")

    def matvec(self, x, y, stream=None):
        """y = x + K gather(x, f2f)."""
        check(lib().hdgx_dense_matvec(self.bs, self.nf, self.nbf, self.K.ptr, self.f2f.ptr, x.ptr, y.ptr,
                                      _stream_ptr(stream)), "hdgx_dense_matvec")

    def workspace(self, restart):
        if restart not in self._ws:
            nb = lib().hdgx_gmres_dense_workspace_bytes(self.bs, self.nf, int(restart))
            self._ws[restart] = torch.empty(int(nb), dtype=torch.uint8, device="cuda")
        return self._ws[restart]

    def gmres(self, x, b=None, restart=20, tol=1e-6, maxit=None, stream=None):
        """kernel/gmres.m on the scaled system (defaults as there: restart 20, tol 1e-6,
        maxit = number of unknowns); x (device, [bs, nf]) is the initial guess and the result.
        Returns (iterations, flag, relres, history)."""
        b = self.F if b is None else b
        maxit = self.bs * self.nf if maxit is None else int(maxit)
        it, fl, rr = ct.c_int(0), ct.c_int(0), ct.c_double(0.0)
        hist = np.zeros(maxit + 1)
        rc = lib().hdgx_gmres_dense(self.bs, self.nf, self.nbf, self.K.ptr, self.f2f.ptr, b.ptr, x.ptr, int(restart),
                                    float(tol), maxit, ct.byref(it), ct.byref(fl), ct.byref(rr),
                                    hist.ctypes.data_as(ct.c_void_p), self.workspace(restart).data_ptr(),
                                    _stream_ptr(stream))
        check(rc, "hdgx_gmres_dense")
        return it.value, fl.value, rr.value, hist[:it.value]
