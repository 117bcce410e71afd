"""CPU checks that pin the oracle and the host set-up to the reference's own numbers.

* master tables vs master/testpython.mat (fixture master_tri_p2.npz);
* oracle flux / fhat vs the reference's generated C kernels (fixture ref_physics.npz);
* oracle schur_uq2 vs the reference MEX sources schur_uq.c (fixture ref_schur.npz).
The fixtures are produced by tests/golden/make_golden.py from the reference tree."""
from pathlib import Path

import numpy as np
import pytest

from hdg_b200.master import mkmaster

G = Path(__file__).resolve().parent / "golden"


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


def test_master_p2_matches_reference_fixture():
    ref = np.load(G / "master_tri_p2.npz")
    m = mkmaster(2, 2, 4)
    for k in ref.files:
        if k in ("nd", "porder"):
            continue
        mine = np.asarray(getattr(m, k), dtype=np.float64)
        r = ref[k]
        assert mine.size == r.size, k
        assert np.abs(mine.reshape(r.shape, order="F") - r).max() < 1e-12, k


@pytest.mark.parametrize("tag", ["ns2d", "ns3d", "euler2d", "euler3d"])
def test_oracle_physics_matches_reference_kernels(oracle, tag):
    d = np.load(G / "ref_physics.npz")
    nd = int(tag[-2])
    p = tag + "_"
    ncu = nd + 2
    f, fu = oracle.flux_points(nd, d[p + "param"], d[p + "udg"])
    fh, fhu, fhh = oracle.fhat_points(nd, d[p + "param"], d[p + "nl"], d[p + "udg"], d[p + "uh"])
    if tag.startswith("euler"):
        # Euler through the (u,q) form (Re = inf): u-parts equal the reference Euler
        # kernels (application/FM/euler), q-parts vanish identically.
        assert np.all(fu[..., ncu:] == 0.0) and np.all(fhu[..., ncu:] == 0.0)
        fu, fhu = fu[..., :ncu], fhu[..., :ncu]
    assert rel(f, d[p + "f"]) < 1e-14
    assert rel(fu, d[p + "f_udg"]) < 1e-14
    assert rel(fh, d[p + "fh"]) < 1e-14
    assert rel(fhu, d[p + "fh_udg"]) < 1e-14
    assert rel(fhh, d[p + "fh_uh"]) < 1e-14


@pytest.mark.parametrize("tag", ["euler2d", "ns2d"])
def test_oracle_schur_matches_reference_mex(oracle, tag):
    d = np.load(G / "ref_schur.npz")
    blk = {k: d[f"{tag}_{k}"] for k in ("M", "C", "E", "BD", "F", "GK", "H", "Rq", "Ru", "Rh")}
    out = oracle.schur_uq(2, blk)
    for k in ("DUDG", "DUDG_DUH", "AE", "FE"):
        assert rel(out[k], d[f"{tag}_uq_{k}"]) < 1e-13, k
