"""hdgx_solve (the Newton loop in native code) against the Python composition of the same C-ABI
calls (hdg_solve) and against the oracle's Newton history."""
import numpy as np
import pytest

from hdg_b200 import configs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ordering", ["mdf", "multicolor"])
def test_native_solve_matches_python_driver(ordering):
    from hdg_b200.solve import hdg_solve, hdgx_solve
    P = configs.c1(n=8)
    U1, H1, r1 = hdgx_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, ordering=ordering)
    U2, H2, r2 = hdg_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, ordering=ordering)
    assert r1["converged"] and r2.converged
    assert r1["iterations"] == r2.iterations
    assert r1["gmres_iters"] == list(r2.gmres_iters)
    assert np.allclose(r1["residuals"], r2.residuals, rtol=1e-9, atol=1e-14)
    assert np.abs(U1 - U2).max() <= 1e-10 * np.abs(U2).max()
    assert np.abs(H1 - H2).max() <= 1e-10 * np.abs(H2).max()


def test_native_solve_ns_matches_oracle_history(oracle):
    from hdg_b200.solve import hdgx_solve
    P = configs.c2(n=6)
    U, H, rep = hdgx_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, tol=1e-10, maxiter=12)
    U_ref, H_ref, res_ref, g_ref, a_ref = oracle.hdg_solve(P, tol=1e-10, maxiter=12)
    assert rep["converged"]
    assert all(abs(a - b) <= 2 for a, b in zip(rep["gmres_iters"], g_ref))
    # Newton is quadratic: compare the history down to the round-off floor
    k = min(len(rep["residuals"]), len(res_ref))
    for a, b in zip(rep["residuals"][:k], res_ref[:k]):
        assert abs(a - b) <= 1e-6 * abs(b) + 1e-12 * res_ref[0]
    assert np.abs(U - U_ref).max() <= 1e-8 * np.abs(U_ref).max()


def test_native_solve_rejects_bad_options():
    from hdg_b200._lib import HdgxError
    from hdg_b200.solve import hdgx_solve
    P = configs.c1(n=3)
    with pytest.raises(HdgxError):
        hdgx_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, restart=0)


@pytest.mark.parametrize("name,kw,mixed", [("c1", dict(n=8), False), ("c2", dict(n=5, porder=3), False),
                                           ("c2", dict(n=5, porder=3), True), ("c4", dict(n=1, porder=3), False)])
def test_graph_captured_assembly_chain_is_bitwise_the_plain_one(name, kw, mixed):
    """On a non-blocking stream hdgx_solve replays its assembly chain (trace gather, elemental
    kernel, block-CSR gather, |F|) from a CUDA graph after the first assembly; on the legacy
    default stream it launches the kernels one by one.  Both give the same bits."""
    import torch
    from hdg_b200.solve import hdgx_solve
    P = configs.by_name(name, **kw)
    U1, H1, r1 = hdgx_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, maxiter=6, mixed=mixed)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        U2, H2, r2 = hdgx_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, maxiter=6, mixed=mixed, stream=s)
    s.synchronize()
    assert r1["iterations"] >= 1 and r1["residuals"] == r2["residuals"]
    # every assembly after the first comes from the graph: at least one per Newton step
    assert r1["graph_assemblies"] == 0 and r2["graph_assemblies"] >= len(r2["residuals"]) - 1
    assert np.array_equal(U1, U2) and np.array_equal(H1, H2)


def test_blocking_host_waits_change_nothing_but_the_wait():
    """hdgx_set_host_wait(1): the host sleeps on blocking-synchronisation events before each
    read-back; the solve's results are the same bits."""
    from hdg_b200._lib import lib
    from hdg_b200.solve import hdgx_solve
    P = configs.c2(n=5, porder=2)
    L = lib()
    prev = L.hdgx_get_host_wait()
    try:
        L.hdgx_set_host_wait(0)
        U0, H0, r0 = hdgx_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, maxiter=6)
        L.hdgx_set_host_wait(1)
        U1, H1, r1 = hdgx_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, maxiter=6)
    finally:
        L.hdgx_set_host_wait(prev)
    assert r0["residuals"] == r1["residuals"] and r0["gmres_iters"] == r1["gmres_iters"]
    assert np.array_equal(U0, U1) and np.array_equal(H0, H1)
