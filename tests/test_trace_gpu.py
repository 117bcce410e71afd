"""GPU parity of the condensed-system path (global assembly, block matvec, BILU(0) factor
and apply, GMRES, back-substitution, Newton) against the CPU oracle.

Tolerances: assembly / matvec / factors / apply / back-substitution 1e-12 relative to the
largest entry (FP64, same ordering); GMRES solutions 1e-8 relative (both stop at a 1e-10
preconditioned residual, so they agree to that tolerance times the conditioning)."""
import numpy as np
import pytest

from hdg_b200 import configs

CASES = [("c1", dict(n=4, porder=2)), ("c2", dict(n=4, porder=3)), ("c4", dict(n=2, porder=2))]


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _setup(oracle, name, kw, ordering="multicolor"):
    from hdg_b200.elemental import DArray
    from hdg_b200.solve import TraceSystem
    P = configs.by_name(name, **kw)
    r = oracle.hdg_elemental(P.master, P.app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    Hg, Rg = oracle.globalassembly(P.mesh, r["AE"], r["FE"], P.master.npf, P.app.ncu)
    ts = TraceSystem(P.mesh, P.master, P.app, ordering=ordering)
    if ordering in ("mdf", "mdf-flags"):
        o2u, u2o = ts.mdf_order(DArray.from_numpy(Hg))
        if ordering == "mdf":
            ts.set_levels(o2u, u2o)
        else:
            ts.set_order(o2u, u2o)
    return P, r, Hg, Rg, ts, DArray


def _order(ts):
    if hasattr(ts, "o2u"):
        return ts.o2u, ts.u2o
    return ts.ord.o2u, ts.ord.u2o


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", CASES)
def test_mdf_order_matches_oracle(oracle, name, kw):
    """The product's MDF order (GPU block norms + host heap) equals the oracle's restatement
    of computeMDFordering.m."""
    P, r, Hg, Rg, ts, DArray = _setup(oracle, name, kw, "mdf")
    o2u_ref, _ = oracle.mdf_ordering(P.mesh, Hg)
    assert np.array_equal(ts.o2u, o2u_ref)


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", CASES)
def test_globalassembly_matvec(oracle, name, kw):
    P, r, Hg, Rg, ts, DArray = _setup(oracle, name, kw)
    dH, dR = ts.empty_blocks(), ts.empty_vec()
    ts.assemble(DArray.from_numpy(r["AE"]), DArray.from_numpy(r["FE"]), dH, dR)
    assert rel(dH.numpy(), Hg) < 1e-14
    assert rel(dR.numpy(), Rg) < 1e-14
    x = np.random.default_rng(0).standard_normal(Rg.shape)
    y = ts.empty_vec()
    ts.matvec(dH, DArray.from_numpy(x), y)
    assert rel(y.numpy(), oracle.matvec(P.mesh, Hg, x)) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("ordering", ["multicolor", "mdf", "mdf-flags"])
@pytest.mark.parametrize("name,kw", CASES)
def test_bilu0_factor_and_apply_same_order(oracle, name, kw, ordering):
    P, r, Hg, Rg, ts, DArray = _setup(oracle, name, kw, ordering)
    o2u, u2o = _order(ts)
    Mg_ref, rc = oracle.bilu0(P.mesh, Hg, o2u, u2o)
    assert rc == 0
    dH, dM = DArray.from_numpy(Hg), ts.empty_blocks()
    ts.bilu0(dH, dM)
    assert rel(dM.numpy(), Mg_ref) < 1e-12
    x = np.random.default_rng(1).standard_normal(Rg.shape)
    v, w = ts.empty_vec(), ts.empty_vec()
    ts.bilu0_apply(dM, DArray.from_numpy(x), v, w)
    assert rel(v.numpy(), oracle.bilu0_apply(P.mesh, Mg_ref, x, o2u, u2o)) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("ordering", ["multicolor", "mdf", "mdf-flags"])
@pytest.mark.parametrize("name,kw", CASES)
def test_gmres_solution(oracle, name, kw, ordering):
    P, r, Hg, Rg, ts, DArray = _setup(oracle, name, kw, ordering)
    o2u, u2o = _order(ts)
    Mg_ref, _ = oracle.bilu0(P.mesh, Hg, o2u, u2o)
    x_ref, flag, it_ref, _ = oracle.gmres_bilu0(P.mesh, Mg_ref, Hg, Rg, np.zeros_like(Rg), o2u, u2o, 20, 1e-10, 1000)
    assert flag == 0
    dH, dM, dR, dx = DArray.from_numpy(Hg), ts.empty_blocks(), DArray.from_numpy(Rg), ts.empty_vec()
    ts.bilu0(dH, dM)
    dx.t.zero_()
    it, fl, rr, hist = ts.gmres(dH, dM, dR, dx, 20, 1e-10, 1000)
    assert fl == 0 and rr <= 1e-10
    assert abs(it - it_ref) <= 2
    x = dx.numpy()
    assert rel(x, x_ref) < 1e-8
    res = oracle.matvec(P.mesh, Hg, x) - Rg
    assert np.linalg.norm(res) / np.linalg.norm(Rg) < 1e-8


@pytest.mark.gpu
def test_backsub(oracle):
    from hdg_b200.elemental import DArray
    from hdg_b200.solve import HDGSolver
    P = configs.c2(n=4, porder=3)
    r = oracle.hdg_elemental(P.master, P.app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    DUH = np.random.default_rng(2).standard_normal((P.app.ncu, P.mesh.nsiz))
    ref = oracle.backsub(P.mesh, r["DUDG"], r["DUDG_DUH"], DUH)
    s = HDGSolver(P.master, P.mesh, P.app)
    s.out.DUDG.t.copy_(DArray.from_numpy(r["DUDG"]).t)
    s.out.DUDG_DUH.t.copy_(DArray.from_numpy(r["DUDG_DUH"]).t)
    s.DUH.t.copy_(DArray.from_numpy(DUH).t)
    s.backsub()
    assert rel(s.DUDGT.numpy(), ref) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", [("c1", dict(n=8)), ("c2", dict(n=6))])
def test_newton_matches_oracle(oracle, name, kw):
    """Same multicolour BILU(0) order on both sides; residual histories agree and both
    converge to |F|/|F0| <= 1e-10."""
    from hdg_b200.solve import hdg_solve
    from hdg_b200.ordering import multicolor
    P = configs.by_name(name, **kw)
    o = multicolor(P.mesh.cbsr_rowpts, P.mesh.cbsr_colind, P.mesh.nf)
    U_ref, H_ref, res_ref, g_ref, a_ref = oracle.hdg_solve(P, o.o2u, o.u2o, tol=1e-10, maxiter=12)
    U, H, rep = hdg_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, tol=1e-10, maxiter=12, ordering=o)
    assert rep.converged and res_ref[-1] / res_ref[0] <= 1e-10
    assert len(rep.residuals) == len(res_ref)
    for a, b in zip(rep.residuals[:-1], res_ref[:-1]):
        assert abs(a - b) <= 1e-6 * max(b, 1e-300) + 1e-12 * res_ref[0]
    assert rel(U, U_ref) < 1e-8 and rel(H, H_ref) < 1e-8


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", [("c1", dict(n=8)), ("c2", dict(n=6)), ("c4", dict(n=2))])
def test_newton_mdf_matches_oracle(oracle, name, kw):
    """Default (MDF-ordered) GPU Newton against the oracle's MDF-ordered Newton."""
    from hdg_b200.solve import hdg_solve
    P = configs.by_name(name, **kw)
    U_ref, H_ref, res_ref, g_ref, a_ref = oracle.hdg_solve(P, tol=1e-10, maxiter=12)
    U, H, rep = hdg_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, tol=1e-10, maxiter=12)
    assert rep.converged
    assert len(rep.residuals) == len(res_ref)
    for a, b in zip(rep.residuals[:-1], res_ref[:-1]):
        assert abs(a - b) <= 1e-6 * max(b, 1e-300) + 1e-12 * res_ref[0]
    for gi, gr in zip(rep.gmres_iters, g_ref):
        assert abs(gi - gr) <= 2
    assert rel(U, U_ref) < 1e-8 and rel(H, H_ref) < 1e-8
