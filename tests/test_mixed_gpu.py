"""Mixed-precision elemental kernel (hdgx_elemental_mixed).

Residual quantities stay FP64: FE (the condensed residual) and DUDG must match the FP64
oracle to 1e-10 relative (the accuracy bound of the mixed form; DUDG with the same ulp-sensitivity
allowance as the FP64 test).  AE and DUDG_DUH are Jacobians computed in FP32 and must match
to 1e-4 relative.  The Newton solve with the mixed kernel must reach |F|/|F0| <= 1e-10 and
agree with the FP64 solve's solution to 1e-9."""
import numpy as np
import pytest

from hdg_b200 import configs

CASES = [("c1", dict(n=4, porder=2)), ("c1", dict(n=3, porder=4)), ("c2", dict(n=4, porder=3)),
         ("c4", dict(n=2, porder=2))]


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", CASES)
def test_mixed_elemental(oracle, name, kw):
    from hdg_b200.elemental import hdg_elemental
    from test_elemental_gpu import ulp_sensitivity
    P = configs.by_name(name, **kw)
    m, a = P.master, P.app
    ref = oracle.hdg_elemental(m, a, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    out = hdg_elemental(m, a, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH, mixed=True)
    assert int(out.status.numpy().max()) == 0
    assert rel(out.FE.numpy(), ref["FE"]) < 1e-10
    assert rel(out.DUDG.numpy(), ref["DUDG"]) < max(1e-10, 10 * ulp_sensitivity(oracle, P))
    assert rel(out.AE.numpy(), ref["AE"]) < 1e-4
    assert rel(out.DUDG_DUH.numpy(), ref["DUDG_DUH"]) < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", [("c1", dict(n=8)), ("c2", dict(n=6))])
def test_mixed_newton_reaches_fp64_solution(name, kw):
    from hdg_b200.solve import hdg_solve
    P = configs.by_name(name, **kw)
    U64, H64, r64 = hdg_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, tol=1e-10, maxiter=16)
    U32, H32, r32 = hdg_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, tol=1e-10, maxiter=16, mixed=True)
    assert r64.converged and r32.converged
    assert r32.residuals[-1] / r32.residuals[0] <= 1e-10
    assert rel(U32, U64) < 1e-9 and rel(H32, H64) < 1e-9
