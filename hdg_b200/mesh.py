"""Simplex meshes and HDG connectivity (host-side set-up, not the hot path).

Restates the reference's mesh pipeline for the square and cube generators:

* ``squaremesh``   -- ``mesh/squaremesh.m`` (triangles, ``parity`` 0/1);
* ``cubemesh``     -- ``mesh/cubemesh.m:29-30`` (6 tets per cube) + ``fixmesh`` orientation
  (``mesh/mkmesh/fixmesh.m``: swap vertices 1,2 of negatively oriented simplices);
* ``mkt2f``        -- ``mesh/mkmesh/mkt2f.m`` (faces numbered in element order, local face
  ``j`` opposite vertex ``j``: ``[[2,3],[3,1],[1,2]]`` / ``[[2,3,4],[1,4,3],[1,2,4],[1,3,2]]``);
* ``setbndnbrs``   -- ``mesh/mkmesh/setbndnbrs.m`` (boundary faces tagged ``-ib``);
* ``reorderface``  -- ``mesh/mkmesh/reorderface.m`` (interior faces first, then boundary
  faces grouped by boundary condition);
* ``createnodes``  -- ``mesh/mkmesh/createnodes.m`` (straight-sided elements);
* ``hdgelcon``     -- ``mesh/mkmesh/elconnectivities.m:147-212`` (``elcon`` by matching
  element face nodes to the face's own nodes);
* ``block_crs``    -- ``mesh/mkmesh/block_crs.m:44-59`` + ``elcon2entcon.m`` (face-row block
  CSR with the diagonal block first in every row).

Index arrays are 1-based, as the reference stores them.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .master import masternodes

_TRI_FACES = np.array([[1, 2], [2, 0], [0, 1]])
_TET_FACES = np.array([[1, 2, 3], [0, 3, 2], [0, 1, 3], [0, 2, 1]])


def squaremesh(m, n, parity=0):
    """``[p, t]`` of an ``m x n``-vertex grid on the unit square, 2 triangles per cell."""
    x, y = np.meshgrid(np.arange(m) / (m - 1), np.arange(n) / (n - 1), indexing="ij")
    p = np.stack([x.ravel(order="F"), y.ravel(order="F")], axis=1)
    if parity == 0:
        t0 = np.array([[1, 2, m + 2], [1, m + 2, m + 1]])
    else:
        t0 = np.array([[1, 2, m + 1], [2, m + 2, m + 1]])
    t = np.kron(t0, np.ones((m - 1, 1), dtype=np.int64)) + np.kron(np.ones_like(t0), np.arange(m - 1)[:, None])
    t = np.kron(t, np.ones((n - 1, 1), dtype=np.int64)) + np.kron(np.ones_like(t), (np.arange(n - 1) * m)[:, None])
    ix = []
    for i in range(1, n):
        ix1 = i + (n - 1) * np.arange(m - 1)
        ix2 = ix1 + (n - 1) * (m - 1)
        ix12 = np.stack([ix2, ix1]) if parity == 0 else np.stack([ix1, ix2])
        ix.extend(ix12.ravel(order="F").tolist())
    t = t[np.array(ix) - 1, :]
    return p, t.astype(np.int64)


def _simplex_volumes(p, t):
    v0 = p[t[:, 0] - 1]
    d = np.stack([p[t[:, k] - 1] - v0 for k in range(1, t.shape[1])], axis=1)
    return np.linalg.det(d)


def cubemesh(m, n, o):
    """``[p, t]`` of an ``m x n x o``-vertex grid on the unit cube, 6 tets per cell."""
    x, y, z = np.meshgrid(np.arange(m) / (m - 1), np.arange(n) / (n - 1), np.arange(o) / (o - 1), indexing="ij")
    p = np.stack([x.ravel(order="F"), y.ravel(order="F"), z.ravel(order="F")], axis=1)
    t0 = np.array([[5, 6, 7, 3], [5, 6, 2, 3], [5, 1, 2, 3], [6, 8, 7, 4], [6, 7, 4, 3], [6, 2, 4, 3]])
    mp = np.array([1, 2])
    mp = np.concatenate([mp, mp + m])
    mp = np.concatenate([mp, mp + m * n])
    t = mp[t0 - 1]
    t = np.kron(t, np.ones((m - 1, 1), dtype=np.int64)) + np.kron(np.ones_like(t), np.arange(m - 1)[:, None])
    t = np.kron(t, np.ones((n - 1, 1), dtype=np.int64)) + np.kron(np.ones_like(t), (np.arange(n - 1) * m)[:, None])
    t = np.kron(t, np.ones((o - 1, 1), dtype=np.int64)) + np.kron(np.ones_like(t), (np.arange(o - 1) * m * n)[:, None])
    flip = _simplex_volumes(p, t) < 0
    t[flip, 0], t[flip, 1] = t[flip, 1].copy(), t[flip, 0].copy()
    return p, t.astype(np.int64)


def mkt2f(t, nd):
    """Faces ``f[nf, nd+2]`` (corners, element 1, element 2 or 0) and ``t2f[nt, nfe]``."""
    faces = _TRI_FACES if nd == 2 else _TET_FACES
    nt, nfv = t.shape
    fv = t[:, faces]                                     # [nt, nfe, nd] vertex ids
    key = np.sort(fv, axis=2).reshape(nt * nfv, nd)
    order = np.lexsort(key.T[::-1])
    ks = key[order]
    same = np.all(ks[1:] == ks[:-1], axis=1)
    nbr = np.full(nt * nfv, -1, dtype=np.int64)          # flat (elem*nfv+j) of the other side
    a = order[:-1][same]
    b = order[1:][same]
    nbr[a] = b
    nbr[b] = a
    t2t = np.where(nbr >= 0, nbr // nfv + 1, 0).reshape(nt, nfv)
    t2f = np.zeros((nt, nfv), dtype=np.int64)
    nbound = int(np.sum(t2t == 0))
    nf = (nfv * nt + nbound) // 2
    f = np.zeros((nf, nd + 2), dtype=np.int64)
    jf = 0
    for i in range(nt):
        for j in range(nfv):
            ie = t2t[i, j]
            if ie > i + 1 or ie <= 0:
                f[jf, :nd] = fv[i, j]
                f[jf, nd] = i + 1
                f[jf, nd + 1] = ie
                jf += 1
                t2f[i, j] = jf
                if ie > 0:
                    k = nbr[i * nfv + j] % nfv
                    t2f[ie - 1, k] = jf
    assert jf == nf
    return f, t2f, t2t


def setbndnbrs(p, f, nd, bndexpr):
    """Tag boundary faces with ``-ib`` for the first predicate that holds on all corners."""
    for ii in np.nonzero(f[:, -1] == 0)[0]:
        pc = p[f[ii, :nd] - 1]
        for jj, ex in enumerate(bndexpr):
            if ex(pc, p):
                f[ii, -1] = -(jj + 1)
                break
        else:
            raise ValueError("Strange boundary.")
    return f


def reorderface(f, t2f, nbc):
    """Interior faces first, then boundary faces ordered by boundary number."""
    nf = f.shape[0]
    inner = np.nonzero(f[:, -1] > 0)[0]
    mp = [inner]
    for ib in range(1, nbc + 1):
        mp.append(np.nonzero(f[:, -1] == -ib)[0])
    mp = np.concatenate(mp)
    f = f[mp]
    a = np.zeros(nf, dtype=np.int64)
    a[mp] = np.arange(1, nf + 1)
    t2f = a[t2f - 1]
    return f, t2f


def createnodes(p, t, plocal):
    """Straight-sided high-order nodes ``dgnodes[npv, nd, ne]``."""
    nd = p.shape[1]
    lam = np.hstack([1.0 - plocal.sum(axis=1, keepdims=True), plocal])   # [npv, nd+1]
    verts = p[t - 1]                                                    # [ne, nd+1, nd]
    dg = np.einsum("pk,ekd->pde", lam, verts)
    return np.ascontiguousarray(dg)


@dataclass
class Mesh:
    nd: int
    porder: int
    p: np.ndarray
    t: np.ndarray
    f: np.ndarray
    t2f: np.ndarray
    perm: np.ndarray
    dgnodes: np.ndarray       # [npv, nd, ne]
    elcon: np.ndarray         # [npf*nfe, ne], 1-based trace node numbers
    bf: np.ndarray            # [nfe, ne]; < 0 marks boundary type -bf
    nsiz: int
    cbsr_rowpts: np.ndarray   # [nf+1], 0-based offsets
    cbsr_colind: np.ndarray   # [nnzb], 1-based face numbers, diagonal first
    bcm_count: int

    @property
    def ne(self):
        return self.t.shape[0]

    @property
    def nf(self):
        return self.f.shape[0]

    @property
    def cbsr_nrows(self):
        return self.nf

    @property
    def cbsr_nblks(self):
        return int(self.cbsr_colind.shape[0])


def hdgelcon(p, f, t2f, dgnodes, perm, porder, nd):
    """elconnectivities.m:147-212: match each element face's nodes to the face's nodes."""
    ne, nfe = t2f.shape
    npf = perm.shape[0]
    _, plocfc, _ = masternodes(porder, nd)
    philocfc = np.hstack([1.0 - plocfc.sum(axis=1, keepdims=True), plocfc])     # [npf, nd]
    snap = 1e-8
    corners = p[f[:, :nd] - 1]                                                  # [nf, nd, nd]
    pf = np.einsum("ak,fkd->fad", philocfc, corners)                            # [nf, npf, nd]
    pf = np.round(pf / snap) * snap
    elcon = np.zeros((npf, nfe, ne), dtype=np.int64)
    dgr = np.round(dgnodes / snap) * snap
    chunk = 8192
    for e0 in range(0, ne, chunk):
        e1 = min(ne, e0 + chunk)
        for j in range(nfe):
            dg = np.transpose(dgr[perm[:, j] - 1, :, e0:e1], (2, 0, 1))           # [c, npf, nd]
            fi = t2f[e0:e1, j] - 1
            pfc = pf[fi]                                                         # [c, npf, nd]
            d2 = np.sum((dg[:, :, None, :] - pfc[:, None, :, :]) ** 2, axis=3)   # [c, a(dg), b(pf)]
            # in(a) = node b of the face matching element face node a (xiny(dg1, pf))
            ib = np.argmin(d2, axis=2)                                           # [c, npf(a)]
            if np.any(np.min(d2, axis=2) > 1e-12):
                raise ValueError("face node matching failed")
            elcon[:, j, e0:e1] = (fi[:, None] * npf + 1 + ib).T
    return elcon.reshape(npf * nfe, ne, order="F")


def block_crs(t2f):
    """Face-to-face block CSR: row i lists ``[i, sorted(other faces sharing an element)]``."""
    ne, nfe = t2f.shape
    nf = int(t2f.max())
    nb = [set() for _ in range(nf)]
    for e in range(ne):
        fs = t2f[e]
        for a in fs:
            nb[a - 1].update(int(x) for x in fs)
    rowpts = np.zeros(nf + 1, dtype=np.int64)
    cols = []
    for i in range(nf):
        s = nb[i]
        s.discard(i + 1)
        row = [i + 1] + sorted(s)
        cols.extend(row)
        rowpts[i + 1] = rowpts[i] + len(row)
    return rowpts, np.array(cols, dtype=np.int64)


def mkf2f(f, t2f):
    """mesh/mkmesh/mkf2f.m: face-to-face connectivity ``f2f[nbf, nf]`` (1-based, 0 = none),
    nbf = 2 nfe - 1.  Column i lists face i, then the other faces of its first element, then
    those of its second element (interior faces only), in local face order."""
    nf = f.shape[0]
    nfe = t2f.shape[1]
    nbf = 2 * nfe - 1
    f2f = np.zeros((nbf, nf), dtype=np.int64)
    t2fa = np.abs(np.asarray(t2f))
    for i in range(nf):
        e1, e2 = int(f[i, -2]), int(f[i, -1])
        k = 0
        f2f[k, i] = i + 1
        for e in ((e1, e2) if e2 > 0 else (e1,)):
            kf = t2fa[e - 1]
            for j in kf:
                if j != i + 1:
                    k += 1
                    f2f[k, i] = j
    return f2f


def mkmesh(p, t, porder, bndexpr, nd):
    """mesh/mkmesh/mkmesh.m + the connectivity part of util/preprocess.m."""
    f, t2f, _ = mkt2f(t, nd)
    f = setbndnbrs(p, f, nd, bndexpr)
    f, t2f = reorderface(f, t2f, len(bndexpr))
    plocal, _, perm = masternodes(porder, nd)
    dgnodes = createnodes(p, t, plocal)
    elcon = hdgelcon(p, f, t2f, dgnodes, perm, porder, nd)
    bf = f[t2f.T - 1, -1]                       # preprocess.m: f(abs(t2f'), end)
    rowpts, colind = block_crs(t2f)
    npf = perm.shape[0]
    return Mesh(nd=nd, porder=porder, p=p, t=t, f=f, t2f=t2f, perm=perm, dgnodes=dgnodes,
                elcon=elcon, bf=bf.astype(np.int64), nsiz=f.shape[0] * npf,
                cbsr_rowpts=rowpts, cbsr_colind=colind, bcm_count=len(bndexpr))


def mkmesh_square(m, n, porder, parity=0, L=1.0, H=1.0):
    """mesh/mkmesh_square.m: boundaries 1 bottom, 2 right, 3 top, 4 left."""
    p, t = squaremesh(m, n, parity)
    p[:, 0] *= L
    p[:, 1] *= H
    bnd = [
        lambda pc, p0: np.all(pc[:, 1] < 1e-6),
        lambda pc, p0: np.all(pc[:, 0] > p0[:, 0].max() - 1e-6),
        lambda pc, p0: np.all(pc[:, 1] > p0[:, 1].max() - 1e-6),
        lambda pc, p0: np.all(pc[:, 0] < 1e-6),
    ]
    return mkmesh(p, t, porder, bnd, 2)


def mkmesh_cube(m, n, o, porder, a=1.0, b=1.0, c=1.0):
    """mesh/mkmesh_cube.m: boundaries x=0, x=a, y=0, y=b, z=0, z=c."""
    p, t = cubemesh(m, n, o)
    p = p * np.array([a, b, c])[None, :]
    bnd = [
        lambda pc, p0: np.all(pc[:, 0] < 1e-6),
        lambda pc, p0: np.all(pc[:, 0] > p0[:, 0].max() - 1e-6),
        lambda pc, p0: np.all(pc[:, 1] < 1e-6),
        lambda pc, p0: np.all(pc[:, 1] > p0[:, 1].max() - 1e-6),
        lambda pc, p0: np.all(pc[:, 2] < 1e-6),
        lambda pc, p0: np.all(pc[:, 2] > p0[:, 2].max() - 1e-6),
    ]
    return mkmesh(p, t, porder, bnd, 3)
