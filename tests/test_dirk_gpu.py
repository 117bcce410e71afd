"""GPU parity of the time-dependent path: the elemental kernel with app.tdep = 1 against the
oracle (same tolerances as the steady elemental tests: 1e-12 on AE, FE, DUDG_DUH, and the
oracle's own one-ulp sensitivity bound on DUDG), getq (hdgx_getq) against the oracle's
restatement of kernel/getq.m, and one DIRK step (hdg_b200.dirk) against the oracle's
restatement of kernel/hdg_solve_dirk.m: each stage is a Newton solve to 1e-10, so the step's
states agree to 1e-8 relative."""
import copy

import numpy as np
import pytest

from hdg_b200 import configs

TOL = 1e-12


def relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _tdep(P, fc_u, seed=4):
    app = copy.copy(P.app)
    app.tdep, app.fc_u = 1, fc_u
    rng = np.random.default_rng(seed)
    SH = np.array(P.SH, copy=True)
    SH[:, :app.ncu, :] = fc_u * P.UDG[:, :app.ncu, :] * (1.0 + 0.1 * rng.standard_normal(SH[:, :app.ncu, :].shape))
    return app, SH


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", [("c1", dict(n=4, porder=2)), ("c2", dict(n=4, porder=3)),
                                     ("c1", dict(n=3, porder=4)), ("c4", dict(n=2, porder=2))])
def test_time_dependent_elemental_matches_oracle(oracle, name, kw):
    from hdg_b200.elemental import hdg_elemental
    P = configs.by_name(name, **kw)
    m, mesh = P.master, P.mesh
    app, SH = _tdep(P, 7.3)
    ref = oracle.hdg_elemental(m, app, mesh.dgnodes, mesh.bf, P.UDG, P.uh_elem(), SH)
    assert ref["nbad"] == 0
    out = hdg_elemental(m, app, mesh.dgnodes, mesh.bf, P.UDG, P.uh_elem(), SH)
    assert int(out.status.numpy().max()) == 0
    for k in ("AE", "FE", "DUDG_DUH"):
        err = relerr(getattr(out, k).numpy(), ref[k])
        assert err < TOL, f"{name} {kw} {k} relerr {err:.3e}"
    rng = np.random.default_rng(7)
    jit = lambda x: x * (1.0 + 2.2e-16 * rng.standard_normal(x.shape))
    ref1 = oracle.hdg_elemental(m, app, jit(mesh.dgnodes), mesh.bf, jit(P.UDG), jit(P.uh_elem()), SH)
    bound = max(TOL, 10.0 * relerr(ref1["DUDG"], ref["DUDG"]))
    err = relerr(out.DUDG.numpy(), ref["DUDG"])
    assert err < bound, f"{name} {kw} DUDG relerr {err:.3e} > {bound:.3e}"
    # the mixed form carries the same terms: its residual FE stays FP64-accurate
    mix = hdg_elemental(m, app, mesh.dgnodes, mesh.bf, P.UDG, P.uh_elem(), SH, mixed=True)
    assert relerr(mix.FE.numpy(), ref["FE"]) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("q,p", [(2, 2), (3, 3)])
def test_dirk_step_matches_oracle(oracle, q, p):
    from hdg_b200.dirk import hdg_solve_dirk
    P = configs.c1(n=4, porder=2)
    dt = 0.05
    Un_ref, Hn_ref = oracle.hdg_solve_dirk(P, 0.0, dt, q, p)
    Un, Hn, reps = hdg_solve_dirk(P.master, P.mesh, P.app, P.UDG, P.UH, 0.0, dt, q, p)
    assert len(reps) == q
    for rep in reps:
        assert rep.residuals[-1] <= 1e-10 * rep.residuals[0]
    assert relerr(Un, Un_ref) < 1e-8
    assert relerr(Hn, Hn_ref) < 1e-8
    # the step moved the state (a time step, not a steady solve)
    assert relerr(Un, np.asarray(P.UDG)) > 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", [("c1", dict(n=4, porder=2)), ("c2", dict(n=4, porder=3)), ("c4", dict(n=2, porder=2))])
def test_getq_matches_oracle(oracle, name, kw):
    """hdgx_getq (kernel/getq.m) against the oracle's restatement, with a q source and fc_q != 1
    and without a source.  Like the q part of DUDG, getq is a small difference of O(1) volume and
    face terms, inv(M) (C u - E uh): the bound is max(1e-12, 10 x the oracle's own change when
    dgnodes, UDG and UH move by one ulp), as for DUDG in the elemental tests."""
    from hdg_b200.elemental import getq
    P = configs.by_name(name, **kw)
    rng = np.random.default_rng(12)
    SH = np.zeros_like(P.UDG)
    SH[:, P.app.ncu:, :] = rng.standard_normal(SH[:, P.app.ncu:, :].shape)
    jit = lambda x: x * (1.0 + 2.2e-16 * rng.standard_normal(x.shape))
    for sh, fc_q in ((SH, 0.7), (None, 1.0)):
        ref = oracle.getq(P.master, P.app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), sh, fc_q)
        ref1 = oracle.getq(P.master, P.app, jit(P.mesh.dgnodes), P.mesh.bf, jit(P.UDG), jit(P.uh_elem()), sh, fc_q)
        bound = max(1e-12, 10.0 * relerr(ref1, ref))
        Q, st = getq(P.master, P.app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), sh, fc_q=fc_q)
        assert int(st.numpy().max()) == 0
        err = relerr(Q.numpy(), ref)
        assert err < bound, f"{name} fc_q={fc_q} relerr {err:.3e} > {bound:.3e}"


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,tdep", [("c1", dict(n=4, porder=2), 0), ("c2", dict(n=4, porder=3), 0),
                                          ("c2", dict(n=4, porder=3), 1), ("c4", dict(n=2, porder=2), 0)])
def test_residual_matches_oracle(oracle, name, kw, tdep):
    """hdgx_residual (kernel/cuda_residual.m: Ru at q = getq(u, uh)) against the oracle's
    restatement.  Ru sums O(1) volume and face terms of a smooth state, so the bound is, as for
    getq and DUDG, max(1e-12, 10 x the oracle's own change under one-ulp input perturbations)."""
    from hdg_b200.elemental import residual
    P = configs.by_name(name, **kw)
    app, SH = (_tdep(P, 7.3) if tdep else (P.app, None))
    rng = np.random.default_rng(21)
    jit = lambda x: x * (1.0 + 2.2e-16 * rng.standard_normal(x.shape))
    ref = oracle.residual(P.master, app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), SH)
    ref1 = oracle.residual(P.master, app, jit(P.mesh.dgnodes), P.mesh.bf, jit(P.UDG), jit(P.uh_elem()), SH)
    bound = max(1e-12, 10.0 * relerr(ref1, ref))
    Ru, st = residual(P.master, app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), SH)
    assert int(st.numpy().max()) == 0
    err = relerr(Ru.numpy(), ref)
    assert err < bound, f"{name} tdep={tdep} relerr {err:.3e} > {bound:.3e}"
