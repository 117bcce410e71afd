"""app.getdqdg = 0 (hdg_elemental.m:20-26, hdg_solve.m:129-132,148-151): the local solve stores
only the u rows of DUDG / DUDG_DUH and the Newton loop recovers q with getq after every update.

* The elemental outputs are exactly the u rows of the getdqdg = 1 outputs (AE, FE unchanged),
  through the device and the host-array entry points.
* The Newton solve matches the oracle's (same residual history to 1e-6, states to 1e-8) and
  converges to the getdqdg = 1 solution (1e-8: the same nonlinear system).
* The native hdgx_solve keeps getdqdg = 1 and refuses 0 with status -2."""
import copy

import numpy as np
import pytest

from hdg_b200 import configs


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _app0(app):
    a = copy.copy(app)
    a.getdqdg = 0
    return a


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", [("c1", dict(n=4, porder=2)), ("c2", dict(n=4, porder=3)), ("c4", dict(n=2, porder=2))])
def test_elemental_stores_the_u_rows(name, kw):
    from hdg_b200.elemental import hdg_elemental, hdg_elemental_host
    P = configs.by_name(name, **kw)
    m, mesh, ncu = P.master, P.mesh, P.app.ncu
    full = hdg_elemental(m, P.app, mesh.dgnodes, mesh.bf, P.UDG, P.uh_elem(), P.SH)
    part = hdg_elemental(m, _app0(P.app), mesh.dgnodes, mesh.bf, P.UDG, P.uh_elem(), P.SH)
    host = hdg_elemental_host(m, _app0(P.app), mesh.dgnodes, mesh.bf, P.UDG, P.uh_elem(), P.SH, chunk=5)
    assert part.DUDG.shape == (m.npv, ncu, mesh.ne) and part.DUDG_DUH.shape[1] == ncu
    for out in (part, host):
        assert np.array_equal(out.AE.numpy(), full.AE.numpy()) and np.array_equal(out.FE.numpy(), full.FE.numpy())
        assert np.array_equal(out.DUDG.numpy(), full.DUDG.numpy()[:, :ncu])
        assert np.array_equal(out.DUDG_DUH.numpy(), full.DUDG_DUH.numpy()[:, :ncu])


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", [("c1", dict(n=4, porder=2)), ("c2", dict(n=4, porder=3))])
def test_newton_with_getq_matches_oracle(oracle, name, kw):
    from hdg_b200.solve import hdg_solve
    P = configs.by_name(name, **kw)
    P0 = copy.copy(P)
    P0.app = _app0(P.app)
    U_ref, H_ref, res_ref, _, _ = oracle.hdg_solve(P0, tol=1e-10, maxiter=12)
    U, H, rep = hdg_solve(P.master, P.mesh, P0.app, P.UDG, P.UH, P.SH, tol=1e-10, maxiter=12)
    assert rep.converged
    assert len(rep.residuals) == len(res_ref)
    for a, b in zip(rep.residuals[:-1], res_ref[:-1]):
        assert abs(a - b) <= 1e-6 * max(b, 1e-300) + 1e-12 * res_ref[0]
    assert rel(U, U_ref) < 1e-8 and rel(H, H_ref) < 1e-8
    U1, H1, rep1 = hdg_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, tol=1e-10, maxiter=12)
    assert rep1.converged
    assert rel(U, U1) < 1e-8 and rel(H, H1) < 1e-8


@pytest.mark.gpu
def test_native_solve_refuses_getdqdg_zero():
    from hdg_b200._lib import HdgxError
    from hdg_b200.solve import hdgx_solve
    P = configs.c1(n=2, porder=1)
    with pytest.raises(HdgxError):
        hdgx_solve(P.master, P.mesh, _app0(P.app), P.UDG, P.UH, P.SH, maxiter=2)
