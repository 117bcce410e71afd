"""Master element tables for simplex HDG elements (host-side set-up, not the hot path).

Restates, in numpy, what the reference builds once per mesh before any element work:

* ``masternodes``  -- ``mesh/mkmesh/masternodes.m:69-184`` (uniform nodes, ``nodetype=0``),
  including ``faceindex`` (``masternodes.m:394-408``);
* ``gaussquad``    -- ``master/gaussquad.m:1-40``; 1D Gauss--Legendre as
  ``master/gaussquad1d.m`` (Golub--Welsch, ``ceil((pgauss-1)/2)+1`` points), tabulated
  triangle / tetrahedron rules from ``master/gaussquad2d.m`` / ``gaussquad3d.m``;
* ``mkshape``      -- ``master/mkshape.m:1-53``: nodal Lagrange bases and their reference
  derivatives.  The reference divides a Koornwinder basis by its Vandermonde matrix; the
  nodal basis is unique, so a centred monomial basis of the same degree gives the same
  functions (to round-off) and is what is used here;
* ``mkmaster``     -- ``master/mkmaster.m:14-96``;
* ``preprocess``   -- ``util/preprocess.m:23-55`` (``shapvt, shapvg, shapvgdotshapvl,
  shapft, shapfg, shapfgdotshapfc``).

All arrays keep MATLAB's shapes and column-major meaning (numpy arrays are indexed the
same way, ``A[i, j, k]`` == ``A(i+1, j+1, k+1)``); ``perm`` is 1-based as in the
reference.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import numpy as np

from . import _quad_tables


# --------------------------------------------------------------------------- nodes
def _trinodes(p):
    """Uniform triangle nodes, ordered as ``ndgrid`` + filter (masternodes.m:84-87)."""
    pts = []
    for j in range(p + 1):          # v (slow)
        for i in range(p + 1):      # u (fast)
            if i + j <= p:
                pts.append((i / p, j / p))
    return np.array(pts, dtype=np.float64)


def _faceindex(p):
    """masternodes.m:394-408: transpose map of the triangular node numbering."""
    n = p + 1
    a = np.zeros((n, n), dtype=np.int64)
    k = 1
    for j in range(n):
        for i in range(n - j):
            a[i, j] = k
            k += 1
    b = a.T
    return b.flatten(order="F")[b.flatten(order="F") > 0] - 1   # 0-based positions


def masternodes(porder, nd):
    """Return ``(plocvl[npv,nd], plocfc[npf,nd-1], perm[npf,nfe])`` with 1-based ``perm``.

    Simplex elements, uniform node distribution (``elemtype=0, nodetype=0``).
    """
    p = int(porder)
    if p < 1:
        raise ValueError("porder must be >= 1")
    if nd == 2:
        ploc = _trinodes(p)
        plocfc = ploc[: p + 1, :1].copy()
        perm = np.zeros((p + 1, 3), dtype=np.int64)
        perm[0] = [p + 1, (p + 1) * (p + 2) // 2, 1]
        for ii in range(2, p + 2):
            perm[ii - 1, 0] = perm[ii - 2, 0] + p + 2 - ii
            perm[ii - 1, 1] = perm[ii - 2, 1] - ii
            perm[ii - 1, 2] = ii
        return ploc, plocfc, perm
    if nd == 3:
        xi = np.linspace(0.0, 1.0, p + 1)
        blocks = [np.hstack([_trinodes(p), np.zeros(((p + 1) * (p + 2) // 2, 1))])]
        for ii in range(p - 1, 0, -1):
            t2 = _trinodes(ii)
            blocks.append(np.hstack([xi[ii] * t2, xi[p - ii] * np.ones((t2.shape[0], 1))]))
        blocks.append(np.array([[0.0, 0.0, 1.0]]))
        ploc = np.vstack(blocks)
        nfc = (p + 1) * (p + 2) // 2
        plocfc = ploc[:nfc, :2].copy()
        pl = ploc.copy()
        pl[np.abs(pl) < 1e-7] = 0.0
        fi = _faceindex(p)
        f1 = np.nonzero(np.abs(pl.sum(axis=1) - 1.0) < 1e-6)[0]
        f2 = np.nonzero(np.abs(pl[:, 0]) < 1e-6)[0][fi]
        f3 = np.nonzero(np.abs(pl[:, 1]) < 1e-6)[0]
        f4 = np.nonzero(np.abs(pl[:, 2]) < 1e-6)[0][fi]
        perm = np.stack([f1, f2, f3, f4], axis=1) + 1
        return ploc, plocfc, perm.astype(np.int64)
    raise ValueError("nd must be 2 or 3")


# ---------------------------------------------------------------------- quadrature
def gaussquad1d(pgauss):
    """Gauss--Legendre on [0,1] with ``ceil((pgauss-1)/2)+1`` points (gaussquad1d.m)."""
    n = int(np.ceil((pgauss - 1) / 2.0)) + 1
    n = max(n, 1)
    x, w = np.polynomial.legendre.leggauss(n)
    return (0.5 * (x + 1.0)).reshape(-1, 1), 0.5 * w


def gaussquad(pgauss, dim):
    if dim == 1:
        return gaussquad1d(pgauss)
    if dim == 2:
        x, w = _quad_tables.TRI[int(pgauss)]
        return np.array(x, dtype=np.float64), np.array(w, dtype=np.float64)
    if dim == 3:
        x, w = _quad_tables.TET[int(pgauss)]
        return np.array(x, dtype=np.float64), np.array(w, dtype=np.float64) / 6.0
    raise ValueError(dim)


# -------------------------------------------------------------------- shape funcs
def _exponents(porder, dim):
    out = []
    for tot in range(porder + 1):
        for e in itertools.product(range(tot + 1), repeat=dim):
            if sum(e) == tot:
                out.append(e)
    return out


def _monomials(pts, exps, centre):
    """Values and first derivatives of centred monomials at ``pts``."""
    x = pts - centre
    npt, dim = x.shape
    nb = len(exps)
    val = np.ones((npt, nb))
    der = np.zeros((dim, npt, nb))
    for k, e in enumerate(exps):
        for d in range(dim):
            val[:, k] *= x[:, d] ** e[d]
        for d in range(dim):
            if e[d] == 0:
                continue
            t = e[d] * x[:, d] ** (e[d] - 1)
            for dd in range(dim):
                if dd != d:
                    t = t * x[:, dd] ** e[dd]
            der[d, :, k] = t
    return val, der


def mkshape(porder, plocal, pts):
    """Nodal shape functions ``nfs[np, npoints, dim+1]`` (mkshape.m:22-53)."""
    plocal = np.asarray(plocal, dtype=np.float64)
    pts = np.asarray(pts, dtype=np.float64)
    dim = plocal.shape[1]
    exps = _exponents(int(porder), dim)
    centre = np.full(dim, 1.0 / (dim + 1))
    A, _ = _monomials(plocal, exps, centre)        # A[node, basis]
    val, der = _monomials(pts, exps, centre)       # val[pt, basis]
    Ainv = np.linalg.inv(A)
    nfs = np.empty((plocal.shape[0], pts.shape[0], dim + 1))
    nfs[:, :, 0] = (val @ Ainv).T
    for d in range(dim):
        nfs[:, :, d + 1] = (der[d] @ Ainv).T
    return nfs


# ------------------------------------------------------------------------ master
@dataclass
class Master:
    nd: int
    porder: int
    pgauss: int
    plocvl: np.ndarray
    plocfc: np.ndarray
    perm: np.ndarray          # [npf, nfe], 1-based
    gpvl: np.ndarray
    gwvl: np.ndarray
    gpfc: np.ndarray
    gwfc: np.ndarray
    shapvl: np.ndarray        # [npv, ngv, nd+1]
    shapfc: np.ndarray        # [npf, ngf, nd]
    shapmv: np.ndarray        # [ngv, npv, nd+1]
    shapmf: np.ndarray        # [ngf, npf, nd]
    shapvt: np.ndarray = field(default=None)
    shapvg: np.ndarray = field(default=None)
    shapvgdotshapvl: np.ndarray = field(default=None)
    shapft: np.ndarray = field(default=None)
    shapfg: np.ndarray = field(default=None)
    shapfgdotshapfc: np.ndarray = field(default=None)

    @property
    def npv(self):
        return self.plocvl.shape[0]

    @property
    def npf(self):
        return self.plocfc.shape[0]

    @property
    def nfe(self):
        return self.perm.shape[1]

    @property
    def ngv(self):
        return self.gpvl.shape[0]

    @property
    def ngf(self):
        return self.gpfc.shape[0]

    @property
    def permgeom(self):
        return self.perm


def mkmaster(nd, porder, pgauss=None):
    """master/mkmaster.m:14-96 followed by util/preprocess.m:23-55."""
    if pgauss is None:
        pgauss = max(2 * porder, 1)
    plocvl, plocfc, perm = masternodes(porder, nd)
    gpvl, gwvl = gaussquad(pgauss, nd)
    gpfc, gwfc = gaussquad(pgauss, nd - 1)
    shapvl = mkshape(porder, plocvl, gpvl)
    shapfc = mkshape(porder, plocfc, gpfc)
    m = Master(nd=nd, porder=porder, pgauss=pgauss, plocvl=plocvl, plocfc=plocfc, perm=perm,
               gpvl=gpvl, gwvl=gwvl, gpfc=gpfc, gwfc=gwfc, shapvl=shapvl, shapfc=shapfc,
               shapmv=np.transpose(shapvl, (1, 0, 2)).copy(),
               shapmf=np.transpose(shapfc, (1, 0, 2)).copy())
    preprocess(m)
    return m


def preprocess(m: Master):
    """util/preprocess.m:23-55: weighted shape tables and their outer products."""
    npv, ngv, nd1 = m.shapvl.shape
    m.shapvt = np.transpose(m.shapvl, (1, 0, 2)).copy()
    m.shapvg = m.shapvl * m.gwvl[None, :, None]
    # shapvgdotshapvl((ii-1)*npv+jj, g, d) = shapvg(jj,g,d) * shapvl(ii,g,1)
    svd = np.einsum("jgd,ig->jigd", m.shapvg, m.shapvl[:, :, 0])
    m.shapvgdotshapvl = svd.reshape(npv * npv, ngv, nd1, order="F")
    npf, ngf, nd = m.shapfc.shape
    m.shapft = np.transpose(m.shapfc, (1, 0, 2)).copy()
    m.shapfg = m.shapfc * m.gwfc[None, :, None]
    sfd = np.einsum("jgd,ig->jigd", m.shapfg, m.shapfc[:, :, 0])
    m.shapfgdotshapfc = sfd.reshape(npf * npf, ngf, nd, order="F")
    return m
