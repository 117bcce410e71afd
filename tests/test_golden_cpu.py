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


# ---------------------------------------------------------------- boundary fluxes (fbou)
def _fbou_tags():
    d = np.load(G / "ref_fbou.npz")
    return sorted({k.rsplit("_ib", 1)[0] for k in d.files if "_ib" in k}), d


@pytest.mark.parametrize("tag", _fbou_tags()[0])
def test_oracle_fbou_matches_reference_kernels(oracle, tag):
    """ns family types 1 (far field), 2 (adiabatic wall), 4 (prescribed pressure) against
    application/FM/ns/fbou_ns{2,3}d.c, euler family type 2 (slip wall) against
    application/FM/euler/fbou_euler{2,3}d.c, with and without the entropy fix."""
    d = _fbou_tags()[1]
    fam = 0 if tag.startswith("ns") else 1
    nd = int(tag[tag.index("d_") - 1])
    g = lambda k: d[f"{tag}_{k}"]
    types = sorted({int(k.split("_ib")[1].split("_")[0]) for k in d.files if k.startswith(tag + "_ib")})
    assert types
    for ib in types:
        fh, fhu, fhh = oracle.fbou_points(fam, nd, ib, g("ub"), g("param"), g("nl"), g("udg"), g("uh"))
        assert rel(fh, g(f"ib{ib}_fh")) < 1e-13, ib
        assert rel(fhu, g(f"ib{ib}_fh_udg")) < 1e-13, ib
        assert rel(fhh, g(f"ib{ib}_fh_uh")) < 1e-13, ib


@pytest.mark.parametrize("nd", [2, 3])
@pytest.mark.parametrize("eps", [0, 1])
def test_oracle_roe_matrices_match_reference(oracle, nd, eps):
    """getan.m absolute 0 (A_n) and 1 (|A_n|, entropy fix when eps > 0) and their derivatives
    against application/FM/getan.c; the fixture's states put |un| below eps c at half the points."""
    d = np.load(G / "ref_fbou.npz")
    tag = f"ns{nd}d_e{eps}"
    g = lambda k: d[f"{tag}_{k}"]
    if eps:
        uh, nl, gam, e = g("uh"), g("nl"), g("param")[0], g("param")[1]
        un = np.einsum("gd,gd->g", uh[:, 1:nd + 1] / uh[:, :1], nl)
        p = (gam - 1) * (uh[:, -1] - 0.5 * (uh[:, 1:nd + 1] ** 2).sum(1) / uh[:, 0])
        c = np.sqrt(gam * p / uh[:, 0])
        assert np.sum(np.abs(un) < e * c) >= 4
    for ab in (0, 1):
        An, Anm = oracle.getan_points(nd, g("param"), ab, g("nl"), g("uh"))
        assert rel(An, g(f"getan{ab}_An")) < 1e-13
        assert rel(Anm, g(f"getan{ab}_Anm")) < 1e-13


def _matlab_fbou(fam, nd, ib, ub, param, nl, udg, uh):
    """Direct numpy transcription of the formulas of the fbou types the generated C kernels do
    not follow: ns/fbou.m case 3 (fbou3d.m case 3) and euler/fbou.m cases 1, 3, 4, 5 with the
    local Lax-Friedrichs scalars of euler/getan.m:25-111."""
    ncu = nd + 2
    gam, eps, minf = param[0], param[1], param[4]
    u = udg[:, :ncu]
    if fam == 0 and ib == 3:
        fh = np.empty_like(uh)
        fh[:, 0] = u[:, 0] - uh[:, 0]
        fh[:, 1:nd + 1] = -uh[:, 1:nd + 1]
        fh[:, -1] = gam * (gam - 1) * minf ** 2 * uh[:, -1] / uh[:, 0] - ub[-1]
        return fh
    if ib == 5:
        uinf = np.tile(ub, (len(uh), 1))
        uinf[:, 0], uinf[:, -1] = u[:, 0], u[:, -1]
        return uinf - uh
    vh = uh[:, 1:nd + 1] / uh[:, :1]
    un = (vh * nl).sum(1)
    p = (gam - 1) * (uh[:, -1] - 0.5 * uh[:, 0] * (vh ** 2).sum(1))
    c = np.sqrt(gam * p / uh[:, 0])
    an = np.abs(un) + c
    if eps > 0:
        an = 0.5 * (an * an / (eps * c) + eps * c)
    An = un - c
    if ib == 1:
        uinf = np.tile(ub, (len(uh), 1))
    else:
        pb = ub[0] if ib == 3 else (ub[-1] - 0.5) * (gam - 1)
        uinf = u.copy()
        uinf[:, -1] = pb / (gam - 1) + 0.5 * (u[:, 1:nd + 1] ** 2).sum(1) / u[:, 0]
    return (an + An)[:, None] * (u - uh) - (an - An)[:, None] * (uinf - uh)


@pytest.mark.parametrize("fam,ib", [(0, 3), (1, 1), (1, 3), (1, 4), (1, 5)])
@pytest.mark.parametrize("nd", [2, 3])
def test_oracle_fbou_matlab_forms(oracle, fam, ib, nd):
    """Types whose generated C departs from the MATLAB fbou.m that hdg_elemental calls: the values
    against the MATLAB formulas, the Jacobians against central differences of the values."""
    from tests.golden.make_golden import fbou_states
    udg, uh, nl, ub = fbou_states(nd, 8, 3 + nd)
    for eps in (0.0, 0.5):
        param = np.array([1.4, eps, 1000.0, 0.72, 0.5, 2.0])
        fh, fhu, fhh = oracle.fbou_points(fam, nd, ib, ub, param, nl, udg, uh)
        assert rel(fh, _matlab_fbou(fam, nd, ib, ub, param, nl, udg, uh)) < 1e-14
        h = 1e-6
        for c in range(udg.shape[1]):
            up, um = udg.copy(), udg.copy()
            up[:, c] += h; um[:, c] -= h
            fd = (_matlab_fbou(fam, nd, ib, ub, param, nl, up, uh) - _matlab_fbou(fam, nd, ib, ub, param, nl, um, uh)) / (2 * h)
            assert np.abs(fhu[:, :, c] - fd).max() <= 1e-6 * max(1.0, np.abs(fd).max()), c
        for c in range(uh.shape[1]):
            hp, hm = uh.copy(), uh.copy()
            hp[:, c] += h; hm[:, c] -= h
            fd = (_matlab_fbou(fam, nd, ib, ub, param, nl, udg, hp) - _matlab_fbou(fam, nd, ib, ub, param, nl, udg, hm)) / (2 * h)
            assert np.abs(fhh[:, :, c] - fd).max() <= 1e-6 * max(1.0, np.abs(fd).max()), c
