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


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", [("c1", dict(n=8)), ("c2", dict(n=6)), ("c4", dict(n=2))])
def test_fp32_preconditioner_gmres_reaches_the_fp64_solution(oracle, name, kw):
    """hdgx_gmres_bilu0_mixed: the same MDF-ordered BILU(0) factors read in FP32 by the level
    sweeps (FP64 sums, FP64 matvec and Arnoldi) solve the FP64 condensed system to the same
    tolerance: the FP64 residual of its solution is at the GMRES tolerance and the solution
    equals the FP64-preconditioned one, with a few iterations more at most."""
    import torch
    from hdg_b200.elemental import DArray
    from hdg_b200.solve import TraceSystem
    P = configs.by_name(name, **kw)
    r = oracle.hdg_elemental(P.master, P.app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    Hg, Rg = oracle.globalassembly(P.mesh, r["AE"], r["FE"], P.master.npf, P.app.ncu)
    ts = TraceSystem(P.mesh, P.master, P.app)
    dH, dR, dM = DArray.from_numpy(Hg), DArray.from_numpy(Rg), ts.empty_blocks()
    ts.bilu0(dH, dM)
    assert ts.bsr.sweep_plan
    x64, x32 = ts.empty_vec(), ts.empty_vec()
    x64.t.zero_()
    x32.t.zero_()
    it64, fl64, _, _ = ts.gmres(dH, dM, dR, x64, 20, 1e-10, 3000)
    Mg32 = torch.empty(dM.t.numel(), dtype=torch.float32, device="cuda")
    it32, fl32, rr32, _ = ts.gmres_mixed(dH, dM, Mg32, dR, x32, 20, 1e-10, 3000)
    assert fl64 == 0 and fl32 == 0 and rr32 <= 1e-10
    assert it32 <= it64 + max(3, it64 // 10)
    assert np.array_equal(Mg32.cpu().numpy(), dM.t.cpu().numpy().astype(np.float32))
    xs = x32.numpy()
    true_res = Rg - oracle.matvec(P.mesh, Hg, xs)
    assert np.linalg.norm(true_res) <= 1e-7 * np.linalg.norm(Rg)
    assert rel(xs, x64.numpy()) < 1e-7
