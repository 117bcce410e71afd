"""The allocation-free GMRES entry point (hdgx_gmres_bilu0_noalloc).

Callers that may not allocate at solve time (a plugin host whose allocator owns every
byte, a latency-critical serving loop, device memory already reserved in arenas) get the
same BILU(0)-preconditioned GMRES with its scratch in an array compiled into the library.
These tests call it twice in a row through the C ABI and compare each result with the
allocating entry point (hdgx_gmres_bilu0) on the same system: for every elimination order
the trace system offers (greedy colours; the minimum-discarded-fill order of
computeMDFordering.m eliminated level by level with single-launch sweeps, which is the
default of hdgx_solve; and the same order with flag-synchronised sweeps).  Both entry points
run one solver implementation, so the iteration counts are equal and the solutions agree
to the 1e-12 relative tolerance of the other trace-system tests (in practice bit for bit).
A system larger than the 16 MiB scratch is refused with status -5 before any GPU work is
queued.  The file name makes pytest collect it last."""
import ctypes as ct

import numpy as np
import pytest

from hdg_b200 import configs


def _system(oracle, ordering):
    from hdg_b200.elemental import DArray
    from hdg_b200.solve import TraceSystem
    P = configs.c1(n=6, porder=2)
    r = oracle.hdg_elemental(P.master, P.app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    Hg, Rg = oracle.globalassembly(P.mesh, r["AE"], r["FE"], P.master.npf, P.app.ncu)
    ts = TraceSystem(P.mesh, P.master, P.app, ordering="multicolor" if ordering == "multicolor" else "mdf")
    dH, dM, dR = DArray.from_numpy(Hg), ts.empty_blocks(), DArray.from_numpy(Rg)
    if ordering == "mdf-flags":
        ts.set_order(*ts.mdf_order(dH))
    ts.bilu0(dH, dM)               # "mdf": MDF order as levels with the single-launch sweep plan
    if ordering == "mdf":
        assert ts.bsr.ncolors > 0 and ts.bsr.sweep_plan
    if ordering == "mdf-flags":
        assert ts.bsr.ncolors == 0 and ts.bsr.sched
    return ts, dH, dM, dR


def _noalloc(ts, dH, dM, dR, x):
    from hdg_b200._lib import lib
    it, fl, rr = ct.c_int(0), ct.c_int(0), ct.c_double(0.0)
    x.t.zero_()
    rc = lib().hdgx_gmres_bilu0_noalloc(ct.byref(ts.bsr), dH.ptr, dM.ptr, dR.ptr, x.ptr, 20, 1e-10, 1000,
                                        ct.byref(it), ct.byref(fl), ct.byref(rr), None, None)
    return rc, it.value, fl.value, rr.value


@pytest.mark.gpu
@pytest.mark.parametrize("ordering", ["multicolor", "mdf", "mdf-flags"])
def test_noalloc_gmres_matches_allocating_entry_point(oracle, ordering):
    ts, dH, dM, dR = _system(oracle, ordering)
    ref = ts.empty_vec()
    ref.t.zero_()
    it_ref, fl_ref, rr_ref, _ = ts.gmres(dH, dM, dR, ref, 20, 1e-10, 1000)   # allocates its workspace
    assert fl_ref == 0
    x_ref = ref.numpy()
    for _ in range(2):
        x = ts.empty_vec()
        rc, it, fl, rr = _noalloc(ts, dH, dM, dR, x)
        assert rc == 0 and fl == 0 and it == it_ref
        err = np.abs(x.numpy() - x_ref).max() / np.abs(x_ref).max()
        assert err < 1e-12, err


@pytest.mark.gpu
def test_noalloc_gmres_rejects_oversize_system():
    from hdg_b200._lib import HdgxBsr, lib
    big = HdgxBsr(10_000_000, 16, 50_000_000, 1, 1, 1, None, 1, 1)   # pointers never touched
    it, fl, rr = ct.c_int(0), ct.c_int(0), ct.c_double(0.0)
    rc = lib().hdgx_gmres_bilu0_noalloc(ct.byref(big), 1, 1, 1, 1, 20, 1e-10, 10, ct.byref(it), ct.byref(fl),
                                        ct.byref(rr), None, None)
    assert rc == -5
    assert b"allocation-free" in lib().hdgx_status_str(-5)
