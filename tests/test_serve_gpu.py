"""Serving: continuous admission of independent solves on per-request streams.

Every request's result in the mix must equal its result alone, bit for bit (the kernels are
deterministic and requests share no reductions); admission under a budget that fits one
request at a time must still complete every request."""
import numpy as np
import pytest


def _mix(seed=3, count=5):
    from hdg_b200.serve import request_mix
    return request_mix(seed, count, nmin=4, nmax=8, pmin=1, pmax=3, rate=50.0)


@pytest.mark.gpu
@pytest.mark.parametrize("ordering,engine", [("multicolor", "native"), ("mdf", "native"), ("mdf", "python")])
def test_results_identical_alone_and_in_mix(ordering, engine):
    # the mix holds several block sizes (p = 1..3), so kernels shared by the requests are
    # launched concurrently with different shared-memory sizes
    from hdg_b200.serve import Server
    alone = _mix()
    Server(slots=1, ordering=ordering, engine=engine).serve_sequential(alone, realtime=False)
    mixed = _mix()
    stats = Server(slots=4, ordering=ordering, engine=engine).serve(mixed, realtime=False)
    assert stats["converged"] == len(mixed)
    for a, b in zip(alone, mixed):
        assert a.error == "" and b.error == ""
        assert a.converged and b.converged
        assert np.array_equal(a.UDG, b.UDG) and np.array_equal(a.UH, b.UH)
        assert a.residuals == b.residuals and a.gmres_iters == b.gmres_iters


@pytest.mark.gpu
def test_admission_under_tight_memory_budget():
    from hdg_b200.serve import Server, footprint_bytes
    reqs = _mix(seed=4, count=4)
    budget = max(footprint_bytes(r.problem) for r in reqs)
    stats = Server(slots=4, memory_budget=budget).serve(reqs, realtime=False)
    assert stats["requests"] == 4 and stats["converged"] == 4
    # with one request's worth of memory, no two solves may overlap
    spans = sorted((r.admitted, r.finished) for r in reqs)
    for (a0, f0), (a1, f1) in zip(spans, spans[1:]):
        assert a1 >= f0 - 1e-3


def _bypass_mix():
    """A small request, then a large one, then two small ones, all queued at t = 0."""
    from hdg_b200.serve import request_mix
    small = request_mix(5, 3, nmin=4, nmax=4, pmin=1, pmax=1, rate=50.0)
    big = request_mix(6, 1, nmin=30, nmax=30, pmin=4, pmax=4, rate=50.0)[0]
    reqs = [small[0], big, small[1], small[2]]
    for i, r in enumerate(reqs):
        r.rid = i
        r.arrival = 1e-3 * i          # this order (the server sorts by arrival, then zeroes it)
    return reqs


@pytest.mark.gpu
@pytest.mark.parametrize("max_bypass", [0, 4])
def test_admission_past_a_request_that_does_not_fit(max_bypass):
    """With memory for the large request alone (or for the small ones together), the small
    requests behind it are admitted while it waits, unless bypassing is switched off."""
    from hdg_b200.serve import Server, footprint_bytes
    reqs = _bypass_mix()
    fp = [footprint_bytes(r.problem) for r in reqs]
    assert fp[0] + fp[2] + fp[3] <= fp[1]
    stats = Server(slots=4, memory_budget=fp[1], max_bypass=max_bypass).serve(reqs, realtime=False)
    assert stats["converged"] == 4
    big, s1 = reqs[1], reqs[2]
    if max_bypass:
        assert s1.admitted < big.admitted
    else:
        assert big.admitted <= s1.admitted
