"""GPU parity of the boundary fluxes (fbou.m) inside the fused elemental kernel.

Every boundary type of both families is exercised on small meshes whose boundary indices
carry different types, against the CPU oracle (whose ns types 1, 2, 4 and Roe matrices are
pinned to the reference's generated C, tests/test_golden_cpu.py), at the elemental
tolerances of tests/test_elemental_gpu.py.  Then the reference drivers' own setting,
bcm = [2, 1] (wall and far field: problem/euler/euler_trefftz.m:31, problem/ns/ns_naca.m:37),
runs a Newton solve on the GPU against the oracle's Newton solve."""
import copy

import numpy as np
import pytest

from hdg_b200 import configs

TOL = 1e-12


def relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _with_bcs(P, bcm, eps=0.0):
    """Copy of problem P with boundary types bcm and boundary states near its freestream."""
    app = copy.deepcopy(P.app)
    nb = len(app.bcm)
    app.bcm = np.array([bcm[i % len(bcm)] for i in range(nb)], dtype=np.int64)
    ub = np.array(app.bcs[0], dtype=np.float64)
    app.bcs = np.array([ub * (1.0 + 0.01 * i) for i in range(nb)])
    app.param = np.array(app.param, dtype=np.float64)
    app.param[1] = eps
    return app


CASES = [
    # (config, kw, fbou types cycled over the boundary indices, entropy-fix width)
    ("c1", dict(n=4, porder=2), (1, 2, 3, 4), 0.0),       # euler family, 2D
    ("c1", dict(n=4, porder=2), (5, 4, 2, 1), 0.3),
    ("c1", dict(n=3, porder=4), (2, 1, 4, 3), 0.0),
    ("c2", dict(n=4, porder=3), (1, 2, 3, 4), 0.0),       # ns family, 2D
    ("c2", dict(n=4, porder=2), (4, 3, 2, 1), 0.5),
    ("c4", dict(n=2, porder=2), (1, 2, 3, 4, 5, 6), 0.0), # euler family, 3D
    ("c4", dict(n=2, porder=1), (2, 1, 4, 3, 6, 5), 0.3),
]


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw,bcm,eps", CASES)
def test_boundary_types_match_oracle(oracle, name, kw, bcm, eps):
    from hdg_b200.elemental import hdg_elemental
    from tests.test_elemental_gpu import ulp_sensitivity
    P = configs.by_name(name, **kw)
    app = _with_bcs(P, bcm, eps)
    Q = copy.copy(P)
    Q.app = app
    ref = oracle.hdg_elemental(P.master, app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    assert ref["nbad"] == 0
    out = hdg_elemental(P.master, app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    assert int(out.status.numpy().max()) == 0
    for k in ("AE", "FE", "DUDG_DUH"):
        err = relerr(getattr(out, k).numpy(), ref[k])
        assert err < TOL, f"{name} {kw} {bcm} {k} relerr {err:.3e}"
    err = relerr(out.DUDG.numpy(), ref["DUDG"])
    bound = max(TOL, 10.0 * ulp_sensitivity(oracle, Q))
    assert err < bound, f"{name} {kw} {bcm} DUDG relerr {err:.3e} > {bound:.3e}"


@pytest.mark.gpu
def test_ns_family_with_boundaries_matches_oracle_3d(oracle):
    """3D Navier-Stokes (fbou3d.m) with far field, adiabatic and isothermal walls and pressure."""
    from hdg_b200.app import make_app
    from hdg_b200.elemental import hdg_elemental
    P = configs.c4(n=2, porder=1)
    app = make_app(3, re=500.0, minf=0.4)
    app.bcm = np.array([1, 2, 3, 4, 1, 2])
    ub = np.array(app.bcs[0])
    app.bcs = np.array([ub * (1.0 + 0.01 * i) for i in range(6)])
    assert app.fbou == "ns"
    ref = oracle.hdg_elemental(P.master, app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    out = hdg_elemental(P.master, app, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH)
    assert ref["nbad"] == 0 and int(out.status.numpy().max()) == 0
    for k in ("AE", "FE", "DUDG_DUH"):
        assert relerr(getattr(out, k).numpy(), ref[k]) < TOL, k


@pytest.mark.gpu
@pytest.mark.parametrize("name,kw", [("c1", dict(n=4, porder=2)), ("c2", dict(n=4, porder=2))])
def test_wall_and_far_field_newton_matches_oracle(oracle, name, kw):
    """bcm = [2, 1] of the reference's drivers: slip or adiabatic walls on two sides, far
    field on the other two; Newton with BILU(0)-GMRES on the GPU against the oracle's."""
    from hdg_b200.solve import hdg_solve
    P = configs.by_name(name, **kw)
    app = copy.deepcopy(P.app)
    app.bcm = np.array([2, 1, 2, 1])
    P.app = app
    U, H, rep = hdg_solve(P.master, P.mesh, app, P.UDG, P.UH, P.SH, tol=1e-10, maxiter=3)
    U_ref, H_ref, res_ref, _, _ = oracle.hdg_solve(P, tol=1e-10, maxiter=3)
    assert len(rep.residuals) == len(res_ref)
    assert rep.residuals[-1] < 0.5 * rep.residuals[0]
    for x, y in zip(rep.residuals[:-1], res_ref[:-1]):
        assert abs(x - y) <= 1e-6 * max(y, 1e-300) + 1e-12 * res_ref[0]
    assert relerr(U, U_ref) < 1e-8 and relerr(H, H_ref) < 1e-8
