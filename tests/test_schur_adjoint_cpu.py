"""CPU pin of the adjoint Schur restatement (oracle.schur_uq_adjoint / schur_u_adjoint, numpy)
against the reference MEX sources kernel/schur_uq_adjoint.c and kernel/schur_u_adjoint.c, through
the committed fixture ref_schur_adjoint.npz (made by tests/golden/make_golden.py from the compiled
reference on the blocks of ref_schur.npz)."""
from pathlib import Path

import numpy as np
import pytest

G = Path(__file__).resolve().parent / "golden"
KEYS = ("DUDG", "DUDG_DUH", "AE", "FE")


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("tag", ["euler2d", "ns2d"])
def test_uq_adjoint_restatement_matches_reference(oracle, tag):
    d, a = np.load(G / "ref_schur.npz"), np.load(G / "ref_schur_adjoint.npz")
    out = oracle.schur_uq_adjoint(*[d[f"{tag}_{k}"] for k in ("M", "C", "E", "BD", "F", "GK", "H", "Rq", "Ru", "Rh")])
    for k, v in zip(KEYS, out):
        assert rel(v, a[f"{tag}_uqadj_{k}"]) < 1e-12, k


@pytest.mark.parametrize("tag", ["euler2d", "ns2d"])
@pytest.mark.parametrize("form", ["uadj", "uadjfull"])
def test_u_adjoint_restatement_matches_reference(oracle, tag, form):
    d, a = np.load(G / "ref_schur.npz"), np.load(G / "ref_schur_adjoint.npz")
    BD, GK = (d[f"{tag}_BDu"], d[f"{tag}_GKu"]) if form == "uadj" else (d[f"{tag}_BD"], d[f"{tag}_GK"])
    out = oracle.schur_u_adjoint(BD, d[f"{tag}_F"], GK, d[f"{tag}_H"], d[f"{tag}_Ru"], d[f"{tag}_Rh"])
    for k, v in zip(KEYS, out):
        ref = a[f"{tag}_{form}_{k}"]
        assert v.shape == ref.shape
        assert rel(v, ref) < 1e-12, k
        assert np.array_equal(v == 0.0, ref == 0.0) or k != "DUDG_DUH"
