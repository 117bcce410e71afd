"""Host-side set-up of the condensed system: elimination order for BILU(0) and the
element -> block gather map of the global assembly.

The reference orders BILU(0) by minimum discarded fill (kernel/computeMDFordering.m), a
strictly sequential order.  On the GPU the rows are coloured so that no two rows of a
colour share a block (greedy colouring of the face graph of block_crs.m); each colour is
then eliminated in one parallel launch.  ILU(0) factors depend on the order, so the
preconditioner (and the GMRES iteration count) differs from the MDF one while the solution
of the linear system does not.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Ordering:
    ncolors: int
    color_ptr: np.ndarray     # [ncolors+1]
    color_rows: np.ndarray    # [nf] rows grouped by colour
    pos: np.ndarray           # [nf] elimination position
    o2u: np.ndarray           # ordered -> unordered (the reference's BILU0ordered2unordered, 0-based)
    u2o: np.ndarray


def multicolor(rowpts, colind, nf):
    """Greedy colouring in natural row order; rows of a colour are mutually non-adjacent."""
    color = np.full(nf, -1, dtype=np.int64)
    for i in range(nf):
        used = set()
        for k in range(rowpts[i] + 1, rowpts[i + 1]):
            c = color[colind[k] - 1]
            if c >= 0:
                used.add(int(c))
        c = 0
        while c in used:
            c += 1
        color[i] = c
    ncol = int(color.max()) + 1
    o2u = np.lexsort((np.arange(nf), color)).astype(np.int32)
    u2o = np.empty(nf, dtype=np.int32)
    u2o[o2u] = np.arange(nf, dtype=np.int32)
    counts = np.bincount(color, minlength=ncol)
    ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    return Ordering(ncol, ptr, o2u.copy(), u2o.copy(), o2u, u2o)


def from_order(o2u):
    """An arbitrary sequential order (e.g. MDF) as one colour per row (for the oracle)."""
    nf = len(o2u)
    o2u = np.asarray(o2u, dtype=np.int32)
    u2o = np.empty(nf, dtype=np.int32)
    u2o[o2u] = np.arange(nf, dtype=np.int32)
    return Ordering(nf, np.arange(nf + 1, dtype=np.int32), o2u.copy(), u2o.copy(), o2u, u2o)


@dataclass
class AssemblyMap:
    blk_e: np.ndarray      # [2*nnzb]
    blk_ab: np.ndarray     # [2*nnzb]  a | b << 8
    blk_row: np.ndarray    # [nnzb]
    face_e: np.ndarray     # [2*nf]
    face_a: np.ndarray     # [2*nf]


def assembly_map(t2f, rowpts, colind):
    """For every block (i, j) the (element, local face of i, local face of j) triples that
    contribute to it (globalassembly.m:24-37 visits them element by element)."""
    ne, nfe = t2f.shape
    nf = len(rowpts) - 1
    nnzb = int(rowpts[-1])
    blk_row = np.repeat(np.arange(nf, dtype=np.int32), np.diff(rowpts))
    blk_e = np.full((nnzb, 2), -1, dtype=np.int32)
    blk_ab = np.zeros((nnzb, 2), dtype=np.int32)
    fill = np.zeros(nnzb, dtype=np.int32)
    face_e = np.full((nf, 2), -1, dtype=np.int32)
    face_a = np.zeros((nf, 2), dtype=np.int32)
    ffill = np.zeros(nf, dtype=np.int32)
    # block index lookup (row, col) -> k
    key = {}
    for i in range(nf):
        for k in range(rowpts[i], rowpts[i + 1]):
            key[(i, int(colind[k]) - 1)] = k
    for e in range(ne):
        fs = t2f[e] - 1
        for a in range(nfe):
            i = int(fs[a])
            face_e[i, ffill[i]] = e
            face_a[i, ffill[i]] = a
            ffill[i] += 1
            for b in range(nfe):
                k = key[(i, int(fs[b]))]
                blk_e[k, fill[k]] = e
                blk_ab[k, fill[k]] = a | (b << 8)
                fill[k] += 1
    assert fill.max() <= 2 and ffill.max() <= 2
    return AssemblyMap(blk_e.ravel(), blk_ab.ravel(), blk_row, face_e.ravel(), face_a.ravel())


def levels_of_order(rowpts, colind, o2u, u2o):
    """Level schedule of a sequential elimination order: level(i) = 1 + max level of the
    neighbours eliminated before i.  ILU(0) factors depend only on which of two coupled
    rows comes first, so eliminating level by level (rows of a level share no block) gives
    exactly the factors of the sequential order.  Returns an Ordering whose "colours" are
    the levels and whose positions are the sequential order's.  Computed by the library's
    hdgx_level_schedule (host code; one pass over the order)."""
    from ._lib import check, lib
    nf = len(o2u)
    rp = np.ascontiguousarray(rowpts, dtype=np.int64)
    ci = np.ascontiguousarray(colind, dtype=np.int32)
    o2u = np.ascontiguousarray(o2u, dtype=np.int32)
    u2o = np.ascontiguousarray(u2o, dtype=np.int32)
    ptr = np.zeros(nf + 1, dtype=np.int32)
    rows = np.zeros(nf, dtype=np.int32)
    nlev = lib().hdgx_level_schedule(nf, rp.ctypes.data, ci.ctypes.data, o2u.ctypes.data, u2o.ctypes.data,
                                     ptr.ctypes.data, rows.ctypes.data)
    if nlev < 0:
        check(nlev, "hdgx_level_schedule")
    return Ordering(nlev, ptr[:nlev + 1].copy(), rows, u2o.copy(), o2u.copy(), u2o.copy())


def sweep_plan(order, rowpts, colind):
    """Flattened level schedule for the single-launch BILU(0) sweeps (hdgx_bsr.sweep_plan):
    [ncolors+1] level offsets, then per slot q of ``order.color_rows`` the record
    (row i, diagonal block rowpts[i], maxd (block, column) pairs of the neighbours eliminated
    before i, maxd pairs of those eliminated after i), -1 padded, 0-based, neighbours in CSR
    order.  Returns (plan int32 array, maxd), or (None, 0) when a row has more than 6
    off-diagonal blocks.  Built by the library's hdgx_sweep_plan (host code)."""
    import ctypes as ct
    from ._lib import check, lib
    rp = np.ascontiguousarray(rowpts, dtype=np.int64)
    ci = np.ascontiguousarray(colind, dtype=np.int32)
    nf = len(rp) - 1
    ptr = np.ascontiguousarray(order.color_ptr, dtype=np.int32)
    rows = np.ascontiguousarray(order.color_rows, dtype=np.int32)
    pos = np.ascontiguousarray(order.pos, dtype=np.int32)
    maxd = ct.c_int(0)
    args = (nf, rp.ctypes.data, ci.ctypes.data, int(order.ncolors), ptr.ctypes.data, rows.ctypes.data, pos.ctypes.data)
    check(lib().hdgx_sweep_plan(*args, None, ct.byref(maxd)), "hdgx_sweep_plan")
    if maxd.value == 0:
        return None, 0
    plan = np.empty(int(order.ncolors) + 1 + nf * (2 + 4 * maxd.value), dtype=np.int32)
    check(lib().hdgx_sweep_plan(*args, plan.ctypes.data, ct.byref(maxd)), "hdgx_sweep_plan")
    return plan, maxd.value
