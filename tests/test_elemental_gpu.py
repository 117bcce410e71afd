"""GPU parity of the fused elemental kernel (hdgx_elemental) against the CPU oracle.

Tolerances (relative to the largest entry of each output):
* AE, FE, DUDG_DUH: 1e-12 (FP64 throughout; the kernel only sums in another order).
* DUDG: the local Newton update is a small difference of O(1) volume and face terms, so
  even the oracle moves by ~5e-12 when its inputs are perturbed by one ulp.  The test
  measures that sensitivity on the same inputs and requires the GPU to stay within
  max(1e-12, 10 x sensitivity)."""
import numpy as np
import pytest

from hdg_b200 import configs

TOL = 1e-12

CASES = [
    ("c1", dict(n=4, porder=1)),
    ("c1", dict(n=4, porder=2)),
    ("c1", dict(n=3, porder=3)),
    ("c1", dict(n=3, porder=4)),
    ("c2", dict(n=4, porder=1)),
    ("c2", dict(n=4, porder=2)),
    ("c2", dict(n=4, porder=3)),
    ("c2", dict(n=3, porder=4)),
    ("c4", dict(n=2, porder=1)),
    ("c4", dict(n=2, porder=2)),
    ("c4", dict(n=2, porder=3)),     # 100 unknowns, 201 right-hand sides: the global-workspace plan
]


def relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def ulp_sensitivity(oracle, P, key="DUDG", seed=7):
    """Relative change of the oracle's `key` when dgnodes/UDG/UH move by ~1 ulp."""
    rng = np.random.default_rng(seed)
    jit = lambda x: x * (1.0 + 2.2e-16 * rng.standard_normal(x.shape))
    r0 = oracle.hdg_elemental(P.master, P.app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    r1 = oracle.hdg_elemental(P.master, P.app, jit(P.mesh.dgnodes), P.mesh.bf, jit(P.UDG), jit(P.uh_elem()), P.SH)
    return relerr(r1[key], r0[key])


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", CASES)
def test_elemental_matches_oracle(oracle, name, kw):
    from hdg_b200.elemental import hdg_elemental
    P = configs.by_name(name, **kw)
    m, a = P.master, P.app
    ref = oracle.hdg_elemental(m, a, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    assert ref["nbad"] == 0
    out = hdg_elemental(m, a, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    assert int(out.status.numpy().max()) == 0
    for k in ("AE", "FE", "DUDG_DUH"):
        err = relerr(getattr(out, k).numpy(), ref[k])
        assert err < TOL, f"{name} {kw} {k} relerr {err:.3e}"
    err = relerr(out.DUDG.numpy(), ref["DUDG"])
    bound = max(TOL, 10.0 * ulp_sensitivity(oracle, P))
    assert err < bound, f"{name} {kw} DUDG relerr {err:.3e} > {bound:.3e}"


@pytest.mark.gpu
def test_elemental_repeatable_and_batch_independent(oracle):
    """Same element, alone or inside a batch, gives bit-identical outputs (one CTA per
    element; no cross-element reductions)."""
    import torch
    from hdg_b200.elemental import hdg_elemental
    P = configs.c2(n=4, porder=3)
    m, a = P.master, P.app
    full = hdg_elemental(m, a, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    again = hdg_elemental(m, a, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    sl = slice(5, 9)
    part = hdg_elemental(m, a, P.mesh.dgnodes[..., sl], P.mesh.bf[:, sl], P.UDG[..., sl],
                         P.uh_elem()[..., sl], P.SH[..., sl])
    for k in ("AE", "FE", "DUDG", "DUDG_DUH"):
        f, g, h = getattr(full, k).numpy(), getattr(again, k).numpy(), getattr(part, k).numpy()
        assert np.array_equal(f, g)
        assert np.array_equal(f[..., sl], h)


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", [("c2", dict(n=4, porder=3)), ("c1", dict(n=4, porder=2))])
def test_curved_elements_match_oracle(oracle, name, kw):
    """Elements with a non-constant jacobian (nodes moved off the straight-sided positions)
    take the general path of the kernel (elimination of the mass matrix per element)."""
    from hdg_b200.elemental import hdg_elemental
    P = configs.by_name(name, **kw)
    m, a = P.master, P.app
    dg = np.array(P.mesh.dgnodes, copy=True)
    x, y = dg[:, 0, :], dg[:, 1, :]
    L = x.max() - x.min()
    dg[:, 0, :] = x + 0.01 * L * np.sin(2 * np.pi * y / L) * np.sin(np.pi * x / L)
    dg[:, 1, :] = y + 0.01 * L * np.sin(2 * np.pi * x / L) * np.sin(np.pi * y / L)
    ref = oracle.hdg_elemental(m, a, dg, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    assert ref["nbad"] == 0
    out = hdg_elemental(m, a, dg, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    assert int(out.status.numpy().max()) == 0
    for k in ("AE", "FE", "DUDG_DUH"):
        err = relerr(getattr(out, k).numpy(), ref[k])
        assert err < TOL, f"curved {name} {k} relerr {err:.3e}"
    err = relerr(out.DUDG.numpy(), ref["DUDG"])
    assert err < max(TOL, 10.0 * ulp_sensitivity(oracle, P)), f"curved {name} DUDG relerr {err:.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("mixed", [False, True])
@pytest.mark.parametrize("chunk", [0, 5, 13, 1000])
def test_host_array_entry_point_matches_device_call(oracle, mixed, chunk):
    """hdgx_elemental_host (host arrays streamed through the GPU in chunks, the last one ragged
    for chunk 5 and 13 on 32 elements; chunk >= ne is one chunk) gives bitwise the outputs of
    the device-array call, which the oracle pins; a singular element's status comes back too."""
    from hdg_b200.elemental import hdg_elemental, hdg_elemental_host
    P = configs.c2(n=4, porder=3)
    m, a = P.master, P.app
    UDG = np.array(P.UDG, copy=True)
    UDG[:, :, 7] = np.nan                                # element 7 reports a failure
    dev = hdg_elemental(m, a, P.mesh.dgnodes, P.mesh.bf, UDG, P.uh_elem(), P.SH, mixed=mixed)
    host = hdg_elemental_host(m, a, P.mesh.dgnodes, P.mesh.bf, UDG, P.uh_elem(), P.SH, mixed=mixed, chunk=chunk)
    assert not host.AE.t.is_cuda
    for k in ("AE", "FE", "DUDG", "DUDG_DUH", "status"):
        assert np.array_equal(getattr(host, k).numpy(), getattr(dev, k).numpy(), equal_nan=True), k
    st = host.status.numpy()
    assert st[7] != 0 and np.all(np.delete(st, 7) == 0)
    if not mixed:                                        # the mixed kernel has its own parity tests
        ref = oracle.hdg_elemental(m, a, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
        keep = np.delete(np.arange(UDG.shape[-1]), 7)
        for k in ("AE", "FE", "DUDG_DUH"):
            assert relerr(getattr(host, k).numpy()[..., keep], ref[k][..., keep]) < TOL, k


@pytest.mark.gpu
def test_host_array_entry_point_rejects_bad_arguments():
    from hdg_b200._lib import lib
    from hdg_b200.elemental import DeviceMaster, app_struct
    import ctypes as ct
    P = configs.c1(n=2, porder=1)
    dm, a = DeviceMaster(P.master), app_struct(P.app)
    buf = np.zeros(64)
    p = buf.ctypes.data
    assert lib().hdgx_elemental_host(ct.byref(dm.c), ct.byref(a), 4, p, p, p, p, p, p, p, p, None, None, 0, 0,
                                     None) == -1
    assert lib().hdgx_elemental_host(ct.byref(dm.c), ct.byref(a), 4, p, p, p, p, p, p, p, p, p, None, 0, -1,
                                     None) == -1
    assert lib().hdgx_elemental_host(ct.byref(dm.c), ct.byref(a), 0, p, p, p, p, p, p, p, p, p, None, 0, 0,
                                     None) == 0


@pytest.mark.gpu
def test_host_array_entry_point_accepts_pageable_memory():
    """hdgx_elemental_host on plain (pageable) numpy buffers through the C ABI: the driver stages
    the copies, the results are still bitwise those of the device call."""
    import ctypes as ct
    from hdg_b200._lib import lib
    from hdg_b200.elemental import DeviceMaster, app_struct, hdg_elemental
    P = configs.c2(n=4, porder=3)
    m, a = P.master, P.app
    dev = hdg_elemental(m, a, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    F = lambda x, t=np.float64: np.ascontiguousarray(np.asarray(x, dtype=t).ravel(order="F"))
    ins = [F(P.mesh.dgnodes), F(P.mesh.bf, np.int32), F(P.UDG), F(P.uh_elem()), F(P.SH)]
    outs = [np.zeros(getattr(dev, k).t.numel()) for k in ("AE", "FE", "DUDG", "DUDG_DUH")]
    st = np.full(P.mesh.ne, -1, dtype=np.int32)
    dm, ac = DeviceMaster(m), app_struct(a)
    rc = lib().hdgx_elemental_host(ct.byref(dm.c), ct.byref(ac), P.mesh.ne, *[x.ctypes.data for x in ins],
                                   *[x.ctypes.data for x in outs], st.ctypes.data, 0, 7, None)
    assert rc == 0
    assert np.all(st == 0)
    for k, o in zip(("AE", "FE", "DUDG", "DUDG_DUH"), outs):
        assert np.array_equal(o, getattr(dev, k).t.cpu().numpy()), k


@pytest.mark.gpu
def test_viscous_tetrahedra_p3_match_oracle(oracle):
    """3D Navier-Stokes at p = 3 (the workspace plan with the viscous terms), Re = 100."""
    from hdg_b200.app import make_app
    from hdg_b200.elemental import hdg_elemental
    P = configs.c4(n=2, porder=3)
    P.app = make_app(3, re=100.0, minf=0.4, tau=2.0)
    m, a = P.master, P.app
    ref = oracle.hdg_elemental(m, a, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    assert ref["nbad"] == 0
    out = hdg_elemental(m, a, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    assert int(out.status.numpy().max()) == 0
    for k in ("AE", "FE", "DUDG_DUH"):
        err = relerr(getattr(out, k).numpy(), ref[k])
        assert err < TOL, f"{k} relerr {err:.3e}"
    err = relerr(out.DUDG.numpy(), ref["DUDG"])
    bound = max(TOL, 10.0 * ulp_sensitivity(oracle, P))
    assert err < bound, f"DUDG relerr {err:.3e} > {bound:.3e}"
