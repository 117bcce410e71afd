"""Shared elemental launches (hdgx_elemental_shared): several independent problems of one
element shape, each with its own physics constants, boundary data and arrays, evaluated in ONE
launch give, bit for bit, the outputs of one hdgx_elemental launch per problem — also with an
odd grid and replayed from a CUDA graph.  The solve combiner (hdgx_solve_combined) batches the
assemblies of concurrent Newton solves this way without changing any solve's result."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _problems(seed, count, p, visc, nmin=3, nmax=6):
    """Requests of one degree and physics kind (request_mix alternates Euler and NS)."""
    from hdg_b200.serve import request_mix
    rs = request_mix(seed, 2 * count, nmin=nmin, nmax=nmax, pmin=p, pmax=p)
    return [r.problem for r in rs if (r.rid % 2 == 1) == visc][:count]


def _same(a, b):
    return all(np.array_equal(x, y) for xa, xb in zip(a, b) for x, y in zip(xa, xb))


def _check_shared(sl):
    def outs():
        return [o for o, it in zip(sl.outputs(), sl.items) if it["ne"] > 0]

    sl.run_each()
    torch.cuda.synchronize()
    ref = outs()
    assert all(int(o[4].max()) == 0 for o in ref)

    def scramble():
        for it in sl.items:
            it["out"].AE.t.fill_(float("nan"))
            it["out"].FE.t.zero_()
            it["out"].DUDG_DUH.t.fill_(float("nan"))

    scramble()
    sl.run()
    torch.cuda.synchronize()
    assert _same(outs(), ref)
    scramble()
    sl.run(grid=7)                     # the schedule changes, not the arithmetic
    torch.cuda.synchronize()
    assert _same(outs(), ref)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        sl.run(stream=torch.cuda.current_stream())
    scramble()
    g.replay()
    torch.cuda.synchronize()
    assert _same(outs(), ref)


@pytest.mark.parametrize("p,visc", [(1, False), (2, True), (3, False), (4, True)])
def test_shared_launch_equals_one_launch_per_problem(p, visc):
    from hdg_b200.batch import SharedLaunch
    _check_shared(SharedLaunch(_problems(11 + p, 5, p, visc)))


def test_shared_launch_tetrahedra():
    from hdg_b200 import configs
    from hdg_b200.batch import SharedLaunch
    from hdg_b200.app import make_app
    probs = [configs.c4(seed=s, n=2) for s in (0, 1, 2)]
    probs[1].app = make_app(3, re=np.inf, minf=0.3, tau=2.0)   # another far-field state
    _check_shared(SharedLaunch(probs))


def test_shared_launch_tetrahedra_p3():
    """Segments on the global-workspace plan (3D p = 3), Euler and NS."""
    from hdg_b200 import configs
    from hdg_b200.app import make_app
    from hdg_b200.batch import SharedLaunch
    for re in (np.inf, 100.0):
        probs = [configs.c4(seed=s, n=1, porder=3) for s in (0, 1, 2)]
        for k, P in enumerate(probs):
            P.app = make_app(3, re=re, minf=0.3 + 0.1 * k, tau=2.0)
        _check_shared(SharedLaunch(probs))


def test_shared_launch_many_segments_and_empty_one():
    """The most segments one launch takes, one of them with no elements."""
    from hdg_b200._lib import lib
    from hdg_b200.batch import SharedLaunch
    nmax = lib().hdgx_elemental_shared_max()
    sl = SharedLaunch(_problems(5, nmax, 2, True, nmin=2, nmax=3))
    assert len(sl.items) == nmax
    sl._arr[3].ne = 0
    sl.items[3]["ne"] = 0
    _check_shared(sl)


@pytest.mark.parametrize("window_us", [0, 200000])
def test_combined_solves_identical_alone_and_in_mix(window_us):
    from hdg_b200.serve import Server, request_mix

    def mk():
        return request_mix(7, 6, nmin=4, nmax=6, pmin=2, pmax=3, rate=50.0)

    alone = mk()
    Server(slots=1, ordering="mdf").serve_sequential(alone, realtime=False)
    mixed = mk()
    srv = Server(slots=6, ordering="mdf", combine=True, window_us=window_us)
    stats = srv.serve(mixed, realtime=False)
    assert stats["converged"] == len(mixed)
    for a, b in zip(alone, mixed):
        assert a.error == "" and b.error == ""
        assert np.array_equal(a.UDG, b.UDG) and np.array_equal(a.UH, b.UH)
        assert a.residuals == b.residuals and a.gmres_iters == b.gmres_iters
    st = srv.combiner_stats
    assert st["submissions"] >= sum(len(r.residuals) for r in mixed)
    assert st["launches"] <= st["submissions"]
    if window_us:
        # with a long window every batch waits for all running solves: assemblies are shared
        assert st["launches"] < st["submissions"]
