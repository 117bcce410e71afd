"""The elemental entry points refuse a master whose table sizes are not those of the compiled
kernel, before any device work.

The kernel is compiled per (nd, porder) for the drivers' quadrature order pgauss = 2 porder
(mkmaster(mesh, 2*porder), problem/euler/euler_trefftz.m:55).  master/mkmaster.m:1 takes
pgauss as a free argument, and a master built with another pgauss has other ngv / ngf: the
kernel would index its tables with the compiled extents.  Every entry point that evaluates
elements returns -3 for such a master.  The check runs on the host before any CUDA call,
so these tests pass dummy (never dereferenced) device pointers and run without a GPU."""
import ctypes as ct

import numpy as np
import pytest

from hdg_b200 import master as hm
from hdg_b200.app import make_app

DUMMY = 16   # a non-null pointer value that the checks never dereference


def _master_c(m):
    from hdg_b200._lib import HdgxMaster
    return HdgxMaster(m.nd, m.porder, m.npv, m.npf, m.nfe, m.ngv, m.ngf, *([DUMMY] * 7))


def _app_c(nd):
    from hdg_b200.elemental import app_struct
    return app_struct(make_app(nd))


def _elemental(fn, mc, ac):
    return fn(ct.byref(mc), ct.byref(ac), 8, *([DUMMY] * 10), None)


@pytest.mark.parametrize("nd,porder", [(2, 1), (2, 2), (2, 3), (2, 4), (3, 1), (3, 2)])
def test_foreign_quadrature_is_refused(nd, porder):
    from hdg_b200._lib import lib
    L = lib()
    m = hm.mkmaster(nd, porder, pgauss=2 * porder + 1 if (nd, porder) != (2, 4) else 7)
    m2 = hm.mkmaster(nd, porder)
    assert (m.ngv, m.ngf) != (m2.ngv, m2.ngf)
    mc, ac = _master_c(m), _app_c(nd)
    assert _elemental(L.hdgx_elemental, mc, ac) == -3
    assert _elemental(L.hdgx_elemental_mixed, mc, ac) == -3
    assert L.hdgx_elemental_host(ct.byref(mc), ct.byref(ac), 8, *([DUMMY] * 10), 0, 0, None) == -3
    assert L.hdgx_getq(ct.byref(mc), ct.byref(ac), 8, *([DUMMY] * 7), None) == -3
    assert L.hdgx_residual(ct.byref(mc), ct.byref(ac), 8, *([DUMMY] * 7), None) == -3
    assert b"pgauss" in L.hdgx_status_str(-3)


def test_foreign_quadrature_is_refused_by_buckets_and_solve():
    from hdg_b200._lib import (HdgxElemBucket, HdgxMesh, HdgxSolveOpts, HdgxSolveReport, lib)
    L = lib()
    bad = _master_c(hm.mkmaster(2, 3, pgauss=7))
    ac = _app_c(2)
    b = HdgxElemBucket(ct.addressof(bad), ct.addressof(ac), 8, *([DUMMY] * 10), 0)
    assert L.hdgx_elemental_buckets(1, ct.byref(b), 0, None) == -3
    rowpts = np.array([0, 1], dtype=np.int64)
    colind = np.array([1], dtype=np.int32)
    t2f = np.ones(3, dtype=np.int32)
    mesh = HdgxMesh(1, 1, DUMMY, DUMMY, DUMMY, t2f.ctypes.data, rowpts.ctypes.data, colind.ctypes.data)
    opts = HdgxSolveOpts(0, 0, 20, 1, 1e-10, 1e-10, 100)
    rep = HdgxSolveReport()
    assert L.hdgx_solve(ct.byref(bad), ct.byref(ac), ct.byref(mesh), DUMMY, DUMMY, DUMMY, ct.byref(opts),
                        ct.byref(rep), None) == -3


@pytest.mark.parametrize("nd,porder,pgauss", [(2, 5, 8), (3, 4, 6)])
def test_uncompiled_degree_is_refused(nd, porder, pgauss):
    from hdg_b200._lib import lib
    m = hm.mkmaster(nd, porder, pgauss=pgauss)
    assert _elemental(lib().hdgx_elemental, _master_c(m), _app_c(nd)) == -3
