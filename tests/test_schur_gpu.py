"""GPU parity of the MEX-layout Schur entry points against the reference MEX sources
(kernel/schur_uq.c, kernel/schur_u.c, kernel/schur_uq_adjoint.c, kernel/schur_u_adjoint.c)
through the committed fixtures ref_schur.npz and ref_schur_adjoint.npz."""
from pathlib import Path

import numpy as np
import pytest

G = Path(__file__).resolve().parent / "golden"


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["euler2d", "ns2d"])
def test_schur_uq_matches_reference_mex(tag):
    from hdg_b200.elemental import schur_uq
    d = np.load(G / "ref_schur.npz")
    args = [d[f"{tag}_{k}"] for k in ("M", "C", "E", "BD", "F", "GK", "H", "Rq", "Ru", "Rh")]
    before = [a.copy() for a in args]
    DUDG, DD, AE, FE, st = schur_uq(*args)
    assert int(st.numpy().max()) == 0
    for k, v in zip(("DUDG", "DUDG_DUH", "AE", "FE"), (DUDG, DD, AE, FE)):
        assert rel(v.numpy(), d[f"{tag}_uq_{k}"]) < 1e-12, k
    for a, b in zip(args, before):
        assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["euler2d", "ns2d"])
def test_schur_u_matches_reference_mex(tag):
    from hdg_b200.elemental import schur_u
    d = np.load(G / "ref_schur.npz")
    DUDG, DD, AE, FE, st = schur_u(d[f"{tag}_BDu"], d[f"{tag}_F"], d[f"{tag}_GKu"], d[f"{tag}_H"],
                                   d[f"{tag}_Ru"], d[f"{tag}_Rh"])
    assert int(st.numpy().max()) == 0
    for k, v in zip(("DUDG", "DUDG_DUH", "AE", "FE"), (DUDG, DD, AE, FE)):
        assert rel(v.numpy(), d[f"{tag}_u_{k}"]) < 1e-12, k


@pytest.mark.gpu
def test_schur_reports_singular_element():
    """A zero mass matrix is reported per element (status 1) instead of faulting."""
    from hdg_b200.elemental import schur_uq
    d = np.load(G / "ref_schur.npz")
    args = {k: d[f"euler2d_{k}"].copy() for k in ("M", "C", "E", "BD", "F", "GK", "H", "Rq", "Ru", "Rh")}
    args["M"][..., 3] = 0.0
    *_, st = schur_uq(*[args[k] for k in ("M", "C", "E", "BD", "F", "GK", "H", "Rq", "Ru", "Rh")])
    s = st.numpy()
    assert s[3] == 1 and np.count_nonzero(s) == 1


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["euler2d", "ns2d"])
def test_schur_uq_adjoint_matches_reference_mex(tag):
    """hdgx_schur_uq_adjoint against kernel/schur_uq_adjoint.c (fixture ref_schur_adjoint.npz)."""
    from hdg_b200.elemental import schur_uq_adjoint
    d, a = np.load(G / "ref_schur.npz"), np.load(G / "ref_schur_adjoint.npz")
    args = [d[f"{tag}_{k}"] for k in ("M", "C", "E", "BD", "F", "GK", "H", "Rq", "Ru", "Rh")]
    before = [x.copy() for x in args]
    DUDG, DD, AE, FE, st = schur_uq_adjoint(*args)
    assert int(st.numpy().max()) == 0
    for k, v in zip(("DUDG", "DUDG_DUH", "AE", "FE"), (DUDG, DD, AE, FE)):
        assert rel(v.numpy(), a[f"{tag}_uqadj_{k}"]) < 1e-12, k
    for x, y in zip(args, before):
        assert np.array_equal(x, y)


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["euler2d", "ns2d"])
@pytest.mark.parametrize("form", ["uadj", "uadjfull"])
def test_schur_u_adjoint_matches_reference_mex(tag, form):
    """hdgx_schur_u_adjoint against kernel/schur_u_adjoint.c, on the D block alone and on the
    full BD / GK (nc > ncu: the packed outputs and their zero tails)."""
    from hdg_b200.elemental import schur_u_adjoint
    d, a = np.load(G / "ref_schur.npz"), np.load(G / "ref_schur_adjoint.npz")
    BD, GK = (d[f"{tag}_BDu"], d[f"{tag}_GKu"]) if form == "uadj" else (d[f"{tag}_BD"], d[f"{tag}_GK"])
    DUDG, DD, AE, FE, st = schur_u_adjoint(BD, d[f"{tag}_F"], GK, d[f"{tag}_H"], d[f"{tag}_Ru"], d[f"{tag}_Rh"])
    assert int(st.numpy().max()) == 0
    for k, v in zip(("DUDG", "DUDG_DUH", "AE", "FE"), (DUDG, DD, AE, FE)):
        ref = a[f"{tag}_{form}_{k}"]
        assert rel(v.numpy(), ref) < 1e-12, k
        assert np.array_equal(v.numpy() == 0.0, ref == 0.0) or k not in ("DUDG", "DUDG_DUH"), k
