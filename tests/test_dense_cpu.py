"""Dense face-block path on the CPU: mkf2f, the oracle's mkDenseBlockSystem / gmres.m restatement,
and the compiled reference arraymul (when built)."""
import numpy as np
import pytest

from hdg_b200 import configs
from hdg_b200.mesh import mkf2f


def _c1_system(oracle, n=4):
    P = configs.c1(n=n)
    m = P.mesh
    o = oracle.hdg_elemental(P.master, P.app, m.dgnodes, m.bf, P.UDG, P.uh_elem(), P.SH, nthreads=4)
    Hg, Rg = oracle.globalassembly(m, o["AE"], o["FE"], P.master.npf, P.app.ncu)
    return P, o, Hg, Rg


def test_mkf2f_lists_the_face_then_its_element_neighbours():
    P = configs.c1(n=3)
    m = P.mesh
    f2f = mkf2f(m.f, m.t2f)
    nfe = m.t2f.shape[1]
    assert f2f.shape == (2 * nfe - 1, m.nf)
    for i in range(m.nf):
        col = f2f[:, i]
        assert col[0] == i + 1
        e1, e2 = m.f[i, -2], m.f[i, -1]
        expect = [j for j in m.t2f[e1 - 1] if j != i + 1]
        if e2 > 0:
            expect += [j for j in m.t2f[e2 - 1] if j != i + 1]
        assert list(col[1:1 + len(expect)]) == expect
        assert np.all(col[1 + len(expect):] == 0)
        # the same faces as the block-CSR row
        rp, ci = m.cbsr_rowpts, m.cbsr_colind
        assert set(col[col > 0]) == set(ci[rp[i]:rp[i + 1]])


def test_oracle_dense_system_is_the_scaled_block_row(oracle):
    P, o, Hg, Rg = _c1_system(oracle)
    m = P.mesh
    f2f, K, F = oracle.dense_block_system(m, o["AE"], o["FE"], P.master.npf, P.app.ncu)
    assert np.array_equal(f2f, mkf2f(m.f, m.t2f))
    rng = np.random.default_rng(0)
    x = rng.standard_normal(Rg.shape)
    y = oracle.dense_matvec(K, f2f, x)
    hx = oracle.matvec(m, Hg, x)
    rp = m.cbsr_rowpts
    for i in range(m.nf):
        D = Hg[:, :, rp[i]]
        assert np.allclose(D @ y[:, i], hx[:, i], rtol=1e-11, atol=1e-11 * np.abs(hx).max())
        assert np.allclose(D @ F[:, i], Rg[:, i], rtol=1e-11, atol=1e-11 * np.abs(Rg).max())


def test_oracle_gmres_dense_solves_the_condensed_system(oracle):
    import scipy.sparse.linalg as spla
    P, o, Hg, Rg = _c1_system(oracle)
    m = P.mesh
    f2f, K, F = oracle.dense_block_system(m, o["AE"], o["FE"], P.master.npf, P.app.ncu)
    x, flag, it, rev = oracle.gmres_dense(K, F, f2f, tol=1e-12, restart=20, maxit=2000)
    assert flag == 0 and rev[-1] <= 1e-12
    # direct solve of the block-CSR system
    bs, nf = Rg.shape
    A = np.zeros((bs * nf, bs * nf))
    rp, ci = m.cbsr_rowpts, m.cbsr_colind
    for i in range(nf):
        for k in range(rp[i], rp[i + 1]):
            j = ci[k] - 1
            A[bs * i:bs * (i + 1), bs * j:bs * (j + 1)] = Hg[:, :, k]
    xd = np.linalg.solve(A, Rg.ravel(order="F")).reshape(bs, nf, order="F")
    assert np.abs(x - xd).max() <= 1e-9 * np.abs(xd).max()


def test_reference_arraymul_gemv_and_gemm(oracle):
    if not oracle.ref_available():
        pytest.skip("compiled reference kernels not built")
    rng = np.random.default_rng(1)
    A = rng.standard_normal((5, 7, 6))
    Bv = rng.standard_normal((7, 6))
    Cv = oracle.ref_mex("arraymul.so", [A, Bv], [(5, 6)])[0]
    assert np.allclose(Cv, np.einsum("rci,ci->ri", A, Bv), rtol=1e-14, atol=1e-14)
    Bm = rng.standard_normal((7, 3, 6))
    Cm = oracle.ref_mex("arraymul.so", [A, Bm], [(5, 3, 6)])[0]
    assert np.allclose(Cm, np.einsum("rki,kci->rci", A, Bm), rtol=1e-14, atol=1e-14)
