"""Edge cases of the elemental and trace-system entry points: empty and single-element
batches, an unsupported boundary type, a non-finite element among finite ones, a zero
right-hand side, and the full-size C2 workload checked on a random sample of elements."""
import copy

import numpy as np
import pytest
import torch

from hdg_b200 import configs

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _sl(P, idx):
    m = P.mesh
    f = lambda a: np.asfortranarray(a[..., idx])
    return f(m.dgnodes), np.asfortranarray(m.bf[:, idx]), f(P.UDG), f(P.uh_elem()), f(P.SH)


def test_empty_and_single_element(oracle):
    from hdg_b200.elemental import hdg_elemental
    P = configs.c2(n=3)
    out = hdg_elemental(P.master, P.app, *_sl(P, np.arange(0)))
    assert out.AE.shape[-1] == 0 and out.AE.t.numel() == 0
    dg, bf, U, H, S = _sl(P, np.array([5]))
    out = hdg_elemental(P.master, P.app, dg, bf, U, H, S)
    ref = oracle.hdg_elemental(P.master, P.app, dg, bf, U, H, S)
    assert int(out.status.numpy()[0]) == 0
    for k in ("AE", "FE", "DUDG_DUH"):
        assert _rel(getattr(out, k).numpy(), ref[k]) < 1e-12


def test_unsupported_boundary_type_is_reported():
    from hdg_b200.elemental import hdg_elemental
    P = configs.c1(n=4)
    app = copy.deepcopy(P.app)
    app.bcm = np.array(app.bcm)
    app.bcm[0] = 9                                  # not a case of euler/fbou.m
    out = hdg_elemental(P.master, app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    st = out.status.numpy()
    touches = np.any(P.mesh.bf == -1, axis=0)       # elements with a face on boundary 1
    assert touches.any()
    assert np.all(st[touches] == 3)
    assert np.all(st[~touches] == 0)


def test_nonfinite_element_does_not_disturb_the_others():
    from hdg_b200.elemental import hdg_elemental
    P = configs.c2(n=4)
    clean = hdg_elemental(P.master, P.app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    U = np.array(P.UDG, copy=True)
    U[:, :, 7] = np.nan
    dirty = hdg_elemental(P.master, P.app, P.mesh.dgnodes, P.mesh.bf, U, P.uh_elem(), P.SH)
    st = dirty.status.numpy()
    assert st[7] != 0
    assert np.all(np.delete(st, 7) == 0)
    keep = np.delete(np.arange(P.mesh.ne), 7)
    for k in ("AE", "FE", "DUDG", "DUDG_DUH"):
        assert np.array_equal(getattr(dirty, k).numpy()[..., keep], getattr(clean, k).numpy()[..., keep])


def test_gmres_zero_rhs_returns_immediately():
    from hdg_b200.elemental import DArray
    from hdg_b200.solve import HDGSolver
    P = configs.c1(n=4)
    s = HDGSolver(P.master, P.mesh, P.app, ordering="multicolor")
    s.assemble(DArray.from_numpy(P.UDG), DArray.from_numpy(P.UH), DArray.from_numpy(P.SH))
    s.ts.bilu0(s.Hg, s.Mg)
    b = s.ts.empty_vec()
    b.t.zero_()
    x = s.ts.empty_vec()
    x.t.zero_()
    it, fl, rr, _ = s.ts.gmres(s.Hg, s.Mg, b, x, 20, 1e-10, 100, s.ws)
    assert it == 0 and fl == 0
    assert float(x.t.abs().max()) == 0.0


def test_full_c2_workload_sampled_against_oracle(oracle):
    """The 32,768-element NS p=3 workload in one launch; 48 random elements against the oracle."""
    from hdg_b200.elemental import hdg_elemental
    P = configs.c2()
    out = hdg_elemental(P.master, P.app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    torch.cuda.synchronize()
    assert int(out.status.numpy().max()) == 0
    idx = np.sort(np.random.default_rng(9).choice(P.mesh.ne, 48, replace=False))
    ref = oracle.hdg_elemental(P.master, P.app, *_sl(P, idx))
    for k in ("AE", "FE", "DUDG_DUH"):
        assert _rel(getattr(out, k).numpy()[..., idx], ref[k]) < 1e-12, k
    # DUDG: bounded by 10x the oracle's own change under a one-ulp perturbation of its inputs
    # (on this mesh the oracle moves by ~7e-10 itself)
    rng = np.random.default_rng(7)
    jit = lambda x: x * (1.0 + 2.2e-16 * rng.standard_normal(x.shape))
    dg, bf, U, H, S = _sl(P, idx)
    ref1 = oracle.hdg_elemental(P.master, P.app, jit(dg), bf, jit(U), jit(H), S)
    sens = _rel(ref1["DUDG"], ref["DUDG"])
    assert _rel(out.DUDG.numpy()[..., idx], ref["DUDG"]) < max(1e-12, 10.0 * sens)
