"""CPU checks of the time-dependent path (kernel/hdg_solve_dirk.m, volint.m:180-221).

* The oracle's time-dependent terms follow volint.m:180-221,241,258 exactly as algebra:
  relative to the steady blocks, Ru gains Mu (SH_u - fc_u u) and the u-u diagonal blocks of BD
  gain fc_u Mu, with Mu = M / fc_q the oracle's own mass matrix (1e-12).
* tdep = 1 with fc_u = 0 and a zero u source leaves every output bit-identical.
* The DIRK tables of the driver equal the oracle's restatement of dirkcoeff and satisfy the
  order conditions of their (stages, order) label."""
import copy

import numpy as np
import pytest

from hdg_b200 import configs

SCHEMES = [(1, 1), (1, 2), (2, 2), (2, 3), (3, 3), (3, 4)]


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _tdep_app(app, fc_u):
    a = copy.copy(app)
    a.tdep, a.fc_u = 1, fc_u
    return a


@pytest.mark.parametrize("name,kw", [("c1", dict(n=3, porder=2)), ("c2", dict(n=3, porder=3))])
def test_oracle_time_dependent_terms_follow_volint(oracle, name, kw):
    P = configs.by_name(name, **kw)
    m, mesh = P.master, P.mesh
    npv, ncu = m.npv, P.app.ncu
    rng = np.random.default_rng(3)
    SH = np.array(P.SH, copy=True)
    SH[:, :ncu, :] = rng.standard_normal(SH[:, :ncu, :].shape)
    fc_u = 2.5
    st = oracle.hdg_elemental(m, P.app, mesh.dgnodes, mesh.bf, P.UDG, P.uh_elem(), SH, intermediates=True)
    td = oracle.hdg_elemental(m, _tdep_app(P.app, fc_u), mesh.dgnodes, mesh.bf, P.UDG, P.uh_elem(), SH,
                              intermediates=True)
    Mu = st["M"] / P.app.fc_q                                   # [npv, npv, ne]
    src = SH[:, :ncu, :] - fc_u * P.UDG[:, :ncu, :]             # nodal values of the source
    dRu = np.einsum("rse,sae->rae", Mu, src)
    assert rel(td["Ru"] - st["Ru"], dRu) < 1e-12
    dBD = td["BD"] - st["BD"]
    want = np.zeros_like(dBD)
    for a in range(ncu):
        want[:, a, :, a, :] = fc_u * Mu
    assert rel(dBD, want) < 1e-12
    for k in ("M", "C", "E", "F", "GK", "H", "Rq", "Rh"):
        assert np.array_equal(td[k], st[k]), k


def test_time_dependent_path_with_zero_coefficients_is_the_steady_path(oracle):
    P = configs.c1(n=3, porder=2)
    m, mesh = P.master, P.mesh
    st = oracle.hdg_elemental(m, P.app, mesh.dgnodes, mesh.bf, P.UDG, P.uh_elem(), P.SH)
    SH = np.array(P.SH, copy=True)
    SH[:, :P.app.ncu, :] = 0.0
    td = oracle.hdg_elemental(m, _tdep_app(P.app, 0.0), mesh.dgnodes, mesh.bf, P.UDG, P.uh_elem(), SH)
    for k in ("AE", "FE", "DUDG", "DUDG_DUH"):
        assert np.array_equal(td[k], st[k]), k


@pytest.mark.parametrize("q,p", SCHEMES)
def test_dirk_tables(oracle, q, p):
    from hdg_b200.dirk import dirk_coefficients
    d, c, t = dirk_coefficients(q, p)
    do, co, to = oracle.dirkcoeff(q, p)
    assert np.allclose(d, do, rtol=0, atol=1e-14) and np.allclose(c, co, rtol=0, atol=1e-14)
    assert np.allclose(t, to, rtol=0, atol=1e-14)
    a = np.linalg.inv(d)
    b = c @ a
    assert np.allclose(np.tril(a), a, atol=1e-15)              # diagonally implicit
    assert np.allclose(a.sum(axis=1), t, atol=1e-9)            # abscissae = row sums
    # order conditions up to the scheme's order (the (3,3) tableau's a1 is given to 10 digits)
    tol = 1e-9
    assert abs(b.sum() - 1.0) < tol
    if p >= 2:
        assert abs(b @ t - 0.5) < tol
    if p >= 3:
        assert abs(b @ t ** 2 - 1.0 / 3.0) < tol
        assert abs(b @ (a @ t) - 1.0 / 6.0) < tol
    if p >= 4:
        assert abs(b @ t ** 3 - 0.25) < tol
        assert abs(b @ (t * (a @ t)) - 1.0 / 8.0) < tol
        assert abs(b @ (a @ t ** 2) - 1.0 / 12.0) < tol
        assert abs(b @ (a @ (a @ t)) - 1.0 / 24.0) < tol


def test_dirk_rejects_unknown_schemes():
    from hdg_b200.dirk import dirk_coefficients
    with pytest.raises(ValueError):
        dirk_coefficients(4, 4)


def _linear_state(P, seed=2):
    """u = a + b x + c y (+ d z) per component, its trace at the face nodes, and -grad u."""
    m, mesh = P.master, P.mesh
    ncu, nd = P.app.ncu, m.nd
    rng = np.random.default_rng(seed)
    coef = rng.standard_normal((nd + 1, ncu))
    x = mesh.dgnodes[:, :nd, :]                                   # [npv, nd, ne]
    UDG = np.zeros_like(P.UDG)
    UDG[:, :ncu, :] = coef[0][None, :, None] + np.einsum("pde,dc->pce", x, coef[1:])
    perm = np.asarray(m.perm) - 1                                 # [npf, nfe] 0-based
    UHe = np.stack([UDG[perm[:, j], :ncu, :] for j in range(perm.shape[1])], axis=0)   # [nfe, npf, ncu, ne]
    UHe = np.ascontiguousarray(UHe.transpose(2, 1, 0, 3)).reshape((ncu, -1, UDG.shape[-1]), order="F")
    grad = np.zeros((m.npv, ncu * nd, UDG.shape[-1]))
    for d in range(nd):
        grad[:, ncu * d:ncu * (d + 1), :] = coef[1 + d][None, :, None]
    return UDG, UHe, grad


@pytest.mark.parametrize("name,kw", [("c1", dict(n=3, porder=2)), ("c4", dict(n=1, porder=2))])
def test_oracle_getq_recovers_minus_the_gradient_of_a_linear_field(oracle, name, kw):
    """getq.m solves M q = C u - E uh; with uh the trace of a linear u this is -grad u exactly."""
    P = configs.by_name(name, **kw)
    UDG, UHe, grad = _linear_state(P)
    Q = oracle.getq(P.master, P.app, P.mesh.dgnodes, P.mesh.bf, UDG, UHe)
    assert rel(Q, -grad) < 1e-11          # an identity up to the round-off of inv(M) (3D: 3e-12)


def test_oracle_getq_zeroes_the_q_equation(oracle):
    P = configs.c2(n=3, porder=3)
    rng = np.random.default_rng(9)
    SH = np.zeros_like(P.UDG)
    SH[:, P.app.ncu:, :] = rng.standard_normal(SH[:, P.app.ncu:, :].shape)
    fc_q = 0.7
    Q = oracle.getq(P.master, P.app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), SH, fc_q)
    U = np.array(P.UDG, copy=True)
    U[:, P.app.ncu:, :] = Q
    a = copy.copy(P.app)
    a.fc_q = fc_q
    blk = oracle.hdg_elemental(P.master, a, P.mesh.dgnodes, P.mesh.bf, U, P.uh_elem(), SH, intermediates=True)
    scale = np.abs(blk["C"]).max() * np.abs(U).max()
    assert np.abs(blk["Rq"]).max() < 1e-12 * scale
