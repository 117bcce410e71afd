"""Argument checks of the shared elemental launch (hdgx_elemental_shared) and of the solve
combiner, which all run on the host before any CUDA call: dummy (never dereferenced) device
pointers, no GPU needed."""
import ctypes as ct

import numpy as np
import pytest

from hdg_b200 import master as hm
from hdg_b200.app import make_app

DUMMY = 16


def _master_c(m):
    from hdg_b200._lib import HdgxMaster
    return HdgxMaster(m.nd, m.porder, m.npv, m.npf, m.nfe, m.ngv, m.ngf, *([DUMMY] * 7))


def _buckets(pairs):
    """pairs: [(master, app)] -> (ctypes bucket array, objects kept alive)."""
    from hdg_b200._lib import HdgxElemBucket
    from hdg_b200.elemental import app_struct
    keep = []
    arr = (HdgxElemBucket * len(pairs))()
    for k, (m, a) in enumerate(pairs):
        mc, ac = _master_c(m), app_struct(a)
        keep += [mc, ac]
        arr[k] = HdgxElemBucket(ct.addressof(mc), ct.addressof(ac), 8, *([DUMMY] * 10), 0)
    return arr, keep


def _shared(arr, n=None, grid=0):
    from hdg_b200._lib import lib
    return lib().hdgx_elemental_shared(len(arr) if n is None else n, ct.cast(arr, ct.c_void_p), grid, None)


def test_limits_and_empty_calls():
    from hdg_b200._lib import lib
    L = lib()
    nmax = L.hdgx_elemental_shared_max()
    assert nmax >= 8
    m = hm.mkmaster(2, 2)
    arr, keep = _buckets([(m, make_app(2, re=100.0))] * (nmax + 1))
    assert _shared(arr) == -5
    assert _shared(arr, n=0) == 0
    assert _shared(arr, n=-1) == -1
    assert _shared(arr, n=2, grid=-1) == -1
    assert L.hdgx_elemental_shared(2, None, 0, None) == -1


@pytest.mark.parametrize("case", ["degree", "physics_kind", "dimension"])
def test_buckets_of_different_kernels_are_refused(case):
    m2 = hm.mkmaster(2, 2)
    if case == "degree":
        pairs = [(m2, make_app(2, re=100.0)), (hm.mkmaster(2, 3), make_app(2, re=100.0))]
    elif case == "physics_kind":
        pairs = [(m2, make_app(2, re=100.0)), (m2, make_app(2, re=np.inf))]
    else:
        pairs = [(m2, make_app(2)), (hm.mkmaster(3, 2), make_app(3))]
    arr, keep = _buckets(pairs)
    assert _shared(arr) == -2


def test_foreign_master_in_any_bucket_is_refused():
    m = hm.mkmaster(2, 2)
    foreign = hm.mkmaster(2, 2, pgauss=5)
    arr, keep = _buckets([(m, make_app(2)), (foreign, make_app(2))])
    assert _shared(arr) == -3


def test_combiner_argument_checks():
    from hdg_b200._lib import lib
    L = lib()
    h = ct.c_void_p()
    assert L.hdgx_combiner_create(-1, ct.byref(h)) == -1
    assert L.hdgx_combiner_create(0, None) == -1
    assert L.hdgx_combiner_destroy(None) == 0
    assert L.hdgx_combiner_stats(None, None, None, None) == -1
    assert L.hdgx_solve_combined(None, None, None, None, None, None, None, None, None, None) == -1
