"""Host-side pieces of the serving loop (no GPU): request generation and footprints."""
import numpy as np

from hdg_b200.serve import FIXED_OVERHEAD, footprint_bytes, request_mix


def test_request_mix_is_seeded_and_poisson():
    a = request_mix(7, 12, nmin=2, nmax=4, pmin=1, pmax=2, rate=20.0)
    b = request_mix(7, 12, nmin=2, nmax=4, pmin=1, pmax=2, rate=20.0)
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert all(np.array_equal(x.problem.UDG, y.problem.UDG) for x, y in zip(a, b))
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)
    assert sum(np.isinf(r.problem.app.param[2]) for r in a) == 6


def test_footprint_grows_with_mesh_and_degree():
    small = request_mix(1, 1, nmin=2, nmax=2, pmin=1, pmax=1)[0]
    big = request_mix(1, 1, nmin=6, nmax=6, pmin=3, pmax=3)[0]
    assert footprint_bytes(big.problem) - FIXED_OVERHEAD > 4 * (footprint_bytes(small.problem) - FIXED_OVERHEAD)
