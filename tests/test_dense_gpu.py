"""Dense face-block path on the GPU against the oracle (mkDenseBlockSystem.m, gmres.m) and
against arraymul.c's semantics (pinned to the compiled reference on the CPU)."""
import numpy as np
import pytest
import torch

from hdg_b200 import configs

pytestmark = pytest.mark.gpu


def _assembled(oracle, name="c1", **kw):
    from hdg_b200.elemental import DArray
    from hdg_b200.solve import HDGSolver
    P = configs.by_name(name, **kw)
    m = P.mesh
    o = oracle.hdg_elemental(P.master, P.app, m.dgnodes, m.bf, P.UDG, P.uh_elem(), P.SH, nthreads=8)
    s = HDGSolver(P.master, m, P.app, ordering="multicolor", denseblock=True)
    s.assemble(DArray.from_numpy(P.UDG), DArray.from_numpy(P.UH), DArray.from_numpy(P.SH))
    torch.cuda.synchronize()
    return P, o, s


def test_arraymul_gemv_and_gemm():
    from hdg_b200.dense import arraymul
    rng = np.random.default_rng(2)
    A = rng.standard_normal((16, 64, 37))
    Bv = rng.standard_normal((64, 37))
    Cv = arraymul(A, Bv).numpy()
    assert np.allclose(Cv, np.einsum("rci,ci->ri", A, Bv), rtol=1e-13, atol=1e-13)
    Bm = rng.standard_normal((64, 5, 37))
    Cm = arraymul(A, Bm).numpy()
    assert Cm.shape == (16, 5, 37)
    assert np.allclose(Cm, np.einsum("rki,kci->rci", A, Bm), rtol=1e-13, atol=1e-13)
    A2 = rng.standard_normal((4, 3))
    B2 = rng.standard_normal((3, 2))
    assert np.allclose(arraymul(A2, B2).numpy()[:, :, 0], A2 @ B2)
    with pytest.raises(Exception):
        arraymul(A, rng.standard_normal((63, 37)))


@pytest.mark.parametrize("name,kw", [("c1", dict(n=6)), ("c2", dict(n=6, porder=2))])
def test_dense_block_system_matches_oracle(oracle, name, kw):
    P, o, s = _assembled(oracle, name, **kw)
    s.dense.build(s.Hg, s.Rg)
    torch.cuda.synchronize()
    assert int(s.dense.status.numpy().max()) == 0
    f2f, K, F = oracle.dense_block_system(P.mesh, s.out.AE.numpy(), s.out.FE.numpy(), P.master.npf, P.app.ncu)
    assert np.array_equal(s.dense.f2f.numpy(), f2f)
    Kg, Fg = s.dense.K.numpy(), s.dense.F.numpy()
    assert np.abs(Kg - K).max() <= 1e-11 * max(1.0, np.abs(K).max())
    assert np.abs(Fg - F).max() <= 1e-11 * max(1.0, np.abs(F).max())
    x = np.random.default_rng(3).standard_normal(F.shape)
    from hdg_b200.elemental import DArray
    dx, dy = DArray.from_numpy(x), DArray.empty(F.shape)
    s.dense.matvec(dx, dy)
    y = oracle.dense_matvec(K, f2f, x)
    assert np.abs(dy.numpy() - y).max() <= 1e-11 * np.abs(y).max()


def test_gmres_dense_matches_oracle(oracle):
    P, o, s = _assembled(oracle, "c1", n=6)
    s.dense.build(s.Hg, s.Rg)
    K, F, f2f = s.dense.K.numpy(), s.dense.F.numpy(), s.dense.f2f.numpy()
    xo, flo, ito, revo = oracle.gmres_dense(K, F, f2f, restart=20, tol=1e-10, maxit=3000)
    s.DUH.t.zero_()
    it, fl, rr, hist = s.dense.gmres(s.DUH, restart=20, tol=1e-10, maxit=3000)
    assert fl == 0 and flo == 0
    assert abs(it - ito) <= 2
    assert np.abs(s.DUH.numpy() - xo).max() <= 1e-8 * np.abs(xo).max()
    # the first residuals follow the oracle's history
    k = min(10, len(hist), len(revo))
    assert np.allclose(hist[:k], revo[:k], rtol=1e-6)


def test_newton_with_dense_block_gmres_converges():
    from hdg_b200.solve import hdg_solve
    P = configs.c1(n=8)
    U, H, rep = hdg_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, tol=1e-10, gmres_tol=1e-12,
                          ordering="multicolor", denseblock=True)
    assert rep.converged
    U2, H2, rep2 = hdg_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, tol=1e-10, gmres_tol=1e-12,
                             ordering="multicolor")
    assert np.abs(U - U2).max() <= 1e-8 * np.abs(U2).max()
