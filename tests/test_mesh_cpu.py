"""Host set-up checks: mesh sizes of the workloads, connectivity and geometry invariants."""
import numpy as np
import pytest

from hdg_b200 import configs
from hdg_b200.master import mkmaster
from hdg_b200.mesh import mkmesh_cube, mkmesh_square


def test_square_mesh_counts_c1():
    m = mkmesh_square(17, 17, 2, 0, 10.0, 10.0)
    assert m.ne == 512 and m.nf == 800 and m.cbsr_nblks == 3872
    assert m.elcon.shape == (9, 512) and m.nsiz == 2400


def test_block_crs_has_diagonal_first():
    m = mkmesh_square(5, 5, 2)
    for i in range(m.nf):
        assert m.cbsr_colind[m.cbsr_rowpts[i]] == i + 1


@pytest.mark.parametrize("mk", [lambda: mkmesh_square(6, 5, 3), lambda: mkmesh_cube(3, 3, 3, 2)])
def test_elcon_shared_nodes_coincide(mk):
    m = mk()
    nd = m.nd
    ms = mkmaster(nd, m.porder)
    npf, nfe = ms.perm.shape
    pos = {}
    for e in range(m.ne):
        for j in range(nfe):
            for a in range(npf):
                x = m.dgnodes[ms.perm[a, j] - 1, :, e]
                k = m.elcon[a + npf * j, e]
                if k in pos:
                    assert np.allclose(pos[k], x, atol=1e-12)
                else:
                    pos[k] = x
    assert len(pos) == m.nsiz


@pytest.mark.parametrize("nd,po", [(2, 1), (2, 3), (3, 1), (3, 2)])
def test_face_normals_point_outward(nd, po):
    """Normals from facegeom's formula (facegeom.m:40-49) point away from the element."""
    m = mkmesh_square(3, 3, po) if nd == 2 else mkmesh_cube(2, 2, 2, po)
    ms = mkmaster(nd, po)
    for e in range(m.ne):
        dg = m.dgnodes[:, :, e]
        cen = dg.mean(axis=0)
        for j in range(ms.nfe):
            pn = dg[ms.perm[:, j] - 1]
            g = 0
            dp = np.stack([ms.shapmf[g, :, k + 1] @ pn for k in range(nd - 1)], axis=1)  # [nd, nd-1]
            if nd == 2:
                nl = np.array([dp[1, 0], -dp[0, 0]])
            else:
                nl = np.cross(dp[:, 0], dp[:, 1])
            fc = ms.shapmf[g, :, 0] @ pn
            assert nl @ (fc - cen) > 0


def test_partition_of_unity_and_quadrature():
    for nd, po in [(2, 1), (2, 2), (2, 3), (2, 4), (3, 1), (3, 2), (3, 3)]:
        ms = mkmaster(nd, po)
        assert np.allclose(ms.shapvl[:, :, 0].sum(axis=0), 1.0, atol=1e-12)
        assert np.allclose(ms.shapvl[:, :, 1:].sum(axis=0), 0.0, atol=1e-10)
        vol = 0.5 if nd == 2 else 1.0 / 6.0
        assert abs(ms.gwvl.sum() - vol) < 1e-12


def test_sweep_plan_records_match_the_level_schedule():
    """Every record lists exactly the row's earlier / later neighbours in CSR order."""
    from hdg_b200.ordering import levels_of_order, sweep_plan
    m = mkmesh_square(6, 6, 2, 0, 1.0, 1.0)
    rp, ci = np.asarray(m.cbsr_rowpts), np.asarray(m.cbsr_colind)
    rng = np.random.default_rng(5)
    o2u = rng.permutation(m.nf).astype(np.int32)
    u2o = np.empty_like(o2u)
    u2o[o2u] = np.arange(m.nf, dtype=np.int32)
    lv = levels_of_order(rp, ci, o2u, u2o)
    plan, maxd = sweep_plan(lv, rp, ci)
    assert maxd == 4
    assert np.array_equal(plan[:lv.ncolors + 1], lv.color_ptr)
    recs = plan[lv.ncolors + 1:].reshape(m.nf, 2 + 4 * maxd)
    for q in range(m.nf):
        i = lv.color_rows[q]
        assert recs[q, 0] == i and recs[q, 1] == rp[i]
        ks = list(range(rp[i] + 1, rp[i + 1]))
        before = [(k, ci[k] - 1) for k in ks if lv.pos[ci[k] - 1] < lv.pos[i]]
        after = [(k, ci[k] - 1) for k in ks if lv.pos[ci[k] - 1] > lv.pos[i]]
        for lst, c0 in ((before, 2), (after, 2 + 2 * maxd)):
            got = recs[q, c0:c0 + 2 * maxd].reshape(maxd, 2)
            assert [tuple(x) for x in got[:len(lst)]] == lst
            assert np.all(got[len(lst):] == -1)


def test_level_schedule_is_the_sequential_orders_wavefront():
    """hdgx_level_schedule: level(i) = 1 + the largest level of the neighbours eliminated
    before i (restated here row by row), rows grouped by level and by position inside a level,
    so that neighbours never share a level; bad permutations are refused."""
    import ctypes as ct
    from hdg_b200._lib import lib
    from hdg_b200.ordering import levels_of_order
    m = mkmesh_square(9, 9, 3, 0, 1.0, 1.0)
    rp, ci = np.asarray(m.cbsr_rowpts), np.asarray(m.cbsr_colind)
    rng = np.random.default_rng(11)
    o2u = rng.permutation(m.nf).astype(np.int32)
    u2o = np.empty_like(o2u)
    u2o[o2u] = np.arange(m.nf, dtype=np.int32)
    lev = np.zeros(m.nf, dtype=np.int64)
    for j in range(m.nf):
        i = o2u[j]
        nb = ci[rp[i] + 1:rp[i + 1]] - 1
        low = nb[u2o[nb] < j]
        lev[i] = lev[low].max() + 1 if low.size else 0
    lv = levels_of_order(rp, ci, o2u, u2o)
    assert lv.ncolors == lev.max() + 1
    want = np.lexsort((u2o, lev))
    assert np.array_equal(lv.color_rows, want)
    assert np.array_equal(np.diff(lv.color_ptr), np.bincount(lev))
    for c in range(lv.ncolors):
        rows = set(lv.color_rows[lv.color_ptr[c]:lv.color_ptr[c + 1]].tolist())
        for i in rows:
            assert not rows & set((ci[rp[i] + 1:rp[i + 1]] - 1).tolist())
    bad = o2u.copy()
    bad[0] = bad[1]
    ptr = np.zeros(m.nf + 1, np.int32)
    out = np.zeros(m.nf, np.int32)
    rp64 = np.ascontiguousarray(rp, np.int64)
    ci32 = np.ascontiguousarray(ci, np.int32)
    assert lib().hdgx_level_schedule(m.nf, rp64.ctypes.data, ci32.ctypes.data, bad.ctypes.data, u2o.ctypes.data,
                                     ptr.ctypes.data, out.ctypes.data) == -1
