"""Master-element tables of every compiled (nd, porder), pinned by what defines them.

The GPU kernel and the oracle read the same host tables, so the tables need pins of their
own beyond the p=2 triangle fixture (master/testpython.mat):

* quadrature (master/gaussquad1d.m, gaussquad2d.m, gaussquad3d.m at pgauss = 2 porder) is exact
  for every monomial of degree <= pgauss on the reference simplex (exact integrals
  a! b! / (a + b + 2)! and a! b! c! / (a + b + c + 3)!);
* the nodal basis (master/mkshape.m) reproduces every polynomial of degree <= porder and its
  gradient at the Gauss points, exactly as a Lagrange basis on plocvl must;
* the weighted and transposed tables of util/preprocess.m:23-55 are what they are defined as;
* perm (the face-to-volume node map) puts the face nodes of face j on the face opposite vertex
  j and carries plocfc onto them through the face's affine map;
* the p=4 face rule and face basis equal those of the quadrilateral p=4 master shipped in
  problem/burgers/results.mat (its faces are the same 1D segments: 5 Gauss points of
  pgauss = 8; the shape values at its own nodes plocfc), fixture master_seg_p4.npz."""
import itertools
from math import factorial
from pathlib import Path

import numpy as np
import pytest

from hdg_b200.master import gaussquad, mkmaster, mkshape

G = Path(__file__).resolve().parent / "golden"
COMPILED = [(2, 1), (2, 2), (2, 3), (2, 4), (3, 1), (3, 2), (3, 3)]


def _exact(exps):
    d = len(exps)
    return float(np.prod([factorial(e) for e in exps]) / factorial(sum(exps) + d))


def _exps(deg, dim):
    return [e for e in itertools.product(range(deg + 1), repeat=dim) if sum(e) <= deg]


@pytest.mark.parametrize("nd,p", COMPILED)
def test_quadrature_exact_to_pgauss(nd, p):
    m = mkmaster(nd, p)
    for x, w, dim in ((m.gpvl, m.gwvl, nd), (m.gpfc, m.gwfc, nd - 1)):
        for e in _exps(m.pgauss, dim):
            val = float(np.sum(w * np.prod(x ** np.array(e)[None, :], axis=1)))
            assert abs(val - _exact(e)) <= 1e-14 * max(1.0, _exact(e)) * 10, (dim, e)


@pytest.mark.parametrize("nd,p", COMPILED)
def test_basis_reproduces_polynomials_and_gradients(nd, p):
    m = mkmaster(nd, p)
    for nodes, pts, shap, dim in ((m.plocvl, m.gpvl, m.shapvl, nd), (m.plocfc, m.gpfc, m.shapfc, nd - 1)):
        for e in _exps(p, dim):
            e = np.array(e)
            q_nodes = np.prod(nodes ** e[None, :], axis=1)
            q_pts = np.prod(pts ** e[None, :], axis=1)
            assert np.abs(shap[:, :, 0].T @ q_nodes - q_pts).max() < 1e-12
            for d in range(dim):
                ed = e.copy()
                if ed[d] == 0:
                    dq = np.zeros(len(pts))
                else:
                    ed[d] -= 1
                    dq = e[d] * np.prod(pts ** ed[None, :], axis=1)
                assert np.abs(shap[:, :, 1 + d].T @ q_nodes - dq).max() < 1e-11, (e, d)
        # Lagrange property: the basis at its own nodes is the identity
        at_nodes = mkshape(p, nodes, nodes)[:, :, 0]
        assert np.abs(at_nodes - np.eye(len(nodes))).max() < 1e-12


@pytest.mark.parametrize("nd,p", COMPILED)
def test_preprocess_tables(nd, p):
    m = mkmaster(nd, p)
    assert np.array_equal(m.shapvt, np.transpose(m.shapvl, (1, 0, 2)))
    assert np.array_equal(m.shapmv, m.shapvt)
    assert np.allclose(m.shapvg, m.shapvl * m.gwvl[None, :, None], rtol=0, atol=0)
    assert np.array_equal(m.shapft, np.transpose(m.shapfc, (1, 0, 2)))
    assert np.allclose(m.shapfg, m.shapfc * m.gwfc[None, :, None], rtol=0, atol=0)
    assert (m.npv, m.npf, m.nfe) == (len(m.plocvl), len(m.plocfc), nd + 1)


@pytest.mark.parametrize("nd,p", COMPILED)
def test_perm_maps_face_nodes_onto_faces(nd, p):
    m = mkmaster(nd, p)
    verts = np.vstack([np.zeros(nd), np.eye(nd)])          # reference simplex
    perm = m.perm - 1
    assert perm.min() >= 0 and perm.max() < m.npv
    for j in range(nd + 1):
        fv = np.delete(verts, j, axis=0)                     # face j: opposite vertex j
        pts = m.plocvl[perm[:, j]]
        # every face node lies on the face's hyperplane
        nrm = np.linalg.svd(np.hstack([fv, np.ones((nd, 1))]))[2][-1]
        assert np.abs(np.hstack([pts, np.ones((len(pts), 1))]) @ nrm).max() < 1e-12
        # and is the image of plocfc under an affine map of the face's vertices
        bary = np.hstack([1.0 - m.plocfc.sum(1, keepdims=True), m.plocfc])
        images = [bary @ fv[list(o)] for o in itertools.permutations(range(nd))]
        assert any(np.abs(im - pts).max() < 1e-12 for im in images), j


def test_p4_face_rule_and_basis_match_reference_master():
    ref = np.load(G / "master_seg_p4.npz")
    x, w = gaussquad(8, 1)
    assert np.abs(x.ravel() - ref["gpfc"].ravel()).max() < 1e-14
    assert np.abs(w.ravel() - ref["gwfc"].ravel()).max() < 1e-14
    m = mkmaster(2, 4)
    assert np.abs(m.gpfc.ravel() - ref["gpfc"].ravel()).max() < 1e-14
    shap = mkshape(4, ref["plocfc"], ref["gpfc"])
    assert np.abs(shap - ref["shapfc"]).max() < 1e-12
