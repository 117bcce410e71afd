"""Serving independent steady HDG solves with continuous admission.

Requests (a mesh, a degree, a physics state) arrive over time.  The server admits a request
as soon as it has arrived, a slot is free and its device footprint (elemental outputs, the
block-CSR matrix and its BILU(0) factors, the Krylov basis, state vectors) fits in the HBM
budget left by the requests already running.  Every admitted request keeps its mesh, master
element and state resident on the device for its whole Newton solve and runs on its own
CUDA stream, so the kernels of different requests overlap on the GPU; slots and memory are
handed to the next waiting request the moment a solve finishes.  Each request's arithmetic
does not depend on what else is running (no cross-request reductions, deterministic
kernels), so a result is the same alone and in the mix.

Latency = completion time - arrival time; throughput = requests / (last completion - first
arrival).  ``serve_sequential`` runs the same requests back to back (one at a time, default
stream) as the reference point.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import configs
from .app import init_udg, inituhat, make_app, state_fourier
from .master import mkmaster
from .mesh import mkmesh_square


@dataclass
class SolveRequest:
    rid: int
    problem: configs.Problem
    arrival: float = 0.0
    tol: float = 1e-10
    maxiter: int = 16
    # filled by the server
    admitted: float = float("nan")
    finished: float = float("nan")
    converged: bool = False
    iterations: int = 0
    residuals: list = field(default_factory=list)
    gmres_iters: list = field(default_factory=list)
    UDG: np.ndarray = None
    UH: np.ndarray = None
    error: str = ""

    @property
    def latency(self):
        return self.finished - self.arrival


FIXED_OVERHEAD = 16 << 20     # master tables, index maps, allocator rounding


def footprint_bytes(problem, restart=20):
    """Device bytes a solve holds: elemental outputs, Hg + Mg, Krylov basis, vectors."""
    m, a, mesh = problem.master, problem.app, problem.mesh
    ne, ncu, nc, npv = mesh.ne, a.ncu, a.nc, m.npv
    ndf = m.npf * m.nfe
    nh, nq = ncu * ndf, npv * nc
    bs = ncu * m.npf
    N = bs * mesh.nf
    elem = 8 * ne * (nh * nh + nh + nq + nq * nh + nq * 3 + ncu * ndf * 2)
    trace = 8 * (2 * bs * bs * int(mesh.cbsr_rowpts[-1]) + N * (restart + 1 + 6))
    return int(1.15 * (elem + trace)) + FIXED_OVERHEAD


def request_mix(seed, count, nmin=8, nmax=24, pmin=1, pmax=4, rate=20.0):
    """Seeded requests: unit square of n x n squares (2 triangles each), degree p, Mach in
    [0.3, 0.8], half inviscid (Euler) and half Navier-Stokes with Re in [200, 2000], state
    = freestream + 1 % smooth velocity perturbation; Poisson arrivals at ``rate`` per second."""
    rng = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    reqs = []
    for rid in range(count):
        t += rng.exponential(1.0 / rate)
        n = int(rng.integers(nmin, nmax + 1))
        p = int(rng.integers(pmin, pmax + 1))
        minf = float(rng.uniform(0.3, 0.8))
        re = np.inf if rid % 2 == 0 else float(rng.uniform(200.0, 2000.0))
        mesh = mkmesh_square(n + 1, n + 1, p, 0, 1.0, 1.0)
        master = mkmaster(2, p, 2 * p)
        app = make_app(2, re=re, minf=minf, tau=2.0)
        u = state_fourier(mesh.dgnodes, 2, 1.4, minf, seed * 1000 + rid, 4, 0.01, "velocity")
        udg = init_udg(u, app.nc)
        uh = inituhat(master.perm, mesh.elcon, udg, app.ncu, mesh.nsiz)
        P = configs.Problem(f"req{rid}", master, mesh, app, udg, uh, np.zeros_like(udg))
        reqs.append(SolveRequest(rid, P, arrival=t))
    return reqs


def _solve_one(req, ordering, mixed, restart, engine="native", combiner=None):
    """One request on the current CUDA stream.  engine "native": one hdgx_solve call (the
    Newton loop and its host-side set-up in the library, which runs without the Python
    interpreter lock, so concurrent requests also overlap on the host), with its elemental
    evaluations batched with the other requests' when a ``combiner`` is given; "python": the
    HDGSolver composition of the same kernels."""
    P = req.problem
    if engine == "native":
        from .solve import hdgx_solve
        U, H, rep = hdgx_solve(P.master, P.mesh, P.app, P.UDG, P.UH, P.SH, tol=req.tol, maxiter=req.maxiter,
                               restart=restart, ordering=ordering, mixed=mixed, combiner=combiner)
        req.UDG, req.UH = U, H
        req.converged, req.iterations = rep["converged"], rep["iterations"]
        req.residuals, req.gmres_iters = list(rep["residuals"]), list(rep["gmres_iters"])
        return
    from .elemental import DArray
    from .solve import HDGSolver
    s = HDGSolver(P.master, P.mesh, P.app, ordering=ordering, restart=restart, mixed=mixed)
    U = DArray.from_numpy(P.UDG)
    H = DArray.from_numpy(P.UH)
    S = DArray.from_numpy(P.SH)
    rep = s.solve(U, H, S, tol=req.tol, maxiter=req.maxiter)
    req.UDG, req.UH = U.numpy(), H.numpy()
    req.converged, req.iterations = rep.converged, rep.iterations
    req.residuals, req.gmres_iters = list(rep.residuals), list(rep.gmres_iters)


def latency_stats(reqs, t0):
    lat = np.array([r.latency for r in reqs])
    end = max(r.finished for r in reqs)
    first = min(r.arrival for r in reqs)
    return {"requests": len(reqs), "converged": int(sum(r.converged for r in reqs)),
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "solves_per_s": len(reqs) / max(end - first, 1e-9),
            "makespan_s": end - first}


class Server:
    def __init__(self, slots=8, memory_budget=None, ordering="multicolor", mixed=False, restart=20, engine="native",
                 max_bypass=4, combine=False, window_us=0, blocking_waits=True):
        """max_bypass: how many later requests may be admitted ahead of a waiting request that
        does not fit yet (a large request waiting for memory does not block small ones behind
        it, but it is not overtaken more than this many times).  combine: the running requests'
        elemental evaluations of one degree and physics kind share launches (native engine,
        FP64; ``solve.Combiner`` with ``window_us``).  blocking_waits: while ``serve`` runs, the
        solves' host threads sleep on blocking-synchronisation events where they wait for the
        GPU (``hdgx_set_host_wait(1)``) instead of each spinning on a core; ``serve_sequential``,
        one solve at a time, keeps the spinning wait."""
        if combine and (engine != "native" or mixed):
            raise ValueError("shared launches need the native engine in FP64")
        if memory_budget is None:
            free, _ = torch.cuda.mem_get_info()
            memory_budget = int(0.8 * free)
        self.slots, self.budget = slots, memory_budget
        self.ordering, self.mixed, self.restart, self.engine = ordering, mixed, restart, engine
        self.max_bypass = max_bypass
        self.combine, self.window_us = combine, window_us
        self.blocking_waits = blocking_waits
        self.combiner_stats = None

    def serve(self, reqs, realtime=True):
        """Run the requests with continuous admission; returns latency statistics."""
        pending = sorted(reqs, key=lambda r: r.arrival)
        lock = threading.Condition()
        state = {"used": 0, "running": 0}
        streams = [torch.cuda.Stream() for _ in range(self.slots)]
        free_streams = list(range(self.slots))
        dev = torch.cuda.current_device()
        combiner = None
        if self.combine:
            from .solve import Combiner
            combiner = Combiner(self.window_us)
        from ._lib import lib
        prev_wait = lib().hdgx_get_host_wait()
        lib().hdgx_set_host_wait(1 if self.blocking_waits else 0)
        try:
            return self._serve(reqs, realtime, pending, lock, state, streams, free_streams, dev, combiner)
        finally:
            lib().hdgx_set_host_wait(prev_wait)

    def _serve(self, reqs, realtime, pending, lock, state, streams, free_streams, dev, combiner):
        t0 = time.perf_counter()
        threads = []

        def now():
            return time.perf_counter() - t0

        def worker(req, sid, fp):
            torch.cuda.set_device(dev)
            try:
                with torch.cuda.stream(streams[sid]):
                    _solve_one(req, self.ordering, self.mixed, self.restart, self.engine, combiner)
                streams[sid].synchronize()
            except Exception as exc:        # a failed request is reported, not fatal
                req.error = repr(exc)
            req.finished = now()
            with lock:
                state["used"] -= fp
                state["running"] -= 1
                free_streams.append(sid)
                lock.notify_all()

        if not realtime:
            for r in pending:
                r.arrival = 0.0
        fps = {r.rid: footprint_bytes(r.problem, self.restart) for r in pending}
        bypassed = {r.rid: 0 for r in pending}

        def pick(t):
            """Index of the request to admit now, or None: the earliest arrived request that
            fits, unless an earlier one that does not fit has been overtaken max_bypass times."""
            if not free_streams:
                return None
            for i, r in enumerate(pending):
                if r.arrival > t:
                    return None
                if state["used"] + fps[r.rid] <= self.budget or state["running"] == 0:
                    return i
                if bypassed[r.rid] >= self.max_bypass:
                    return None
            return None

        while pending:
            with lock:
                while True:
                    t = now()
                    i = pick(t)
                    if i is not None:
                        break
                    nxt = [r.arrival - t for r in pending if r.arrival > t]
                    lock.wait(timeout=max(1e-3, min(min(nxt), 0.05)) if nxt else 0.05)
                req = pending.pop(i)
                for r in pending[:i]:
                    bypassed[r.rid] += 1
                fp = fps[req.rid]
                sid = free_streams.pop(0)
                state["used"] += fp
                state["running"] += 1
            req.admitted = now()
            th = threading.Thread(target=worker, args=(req, sid, fp), daemon=True)
            th.start()
            threads.append(th)
        for th in threads:
            th.join()
        if combiner is not None:
            self.combiner_stats = combiner.stats()
            combiner.close()
        return latency_stats(reqs, t0)

    def serve_sequential(self, reqs, realtime=True):
        """Back-to-back plain solves: one request at a time, in arrival order."""
        t0 = time.perf_counter()
        for req in sorted(reqs, key=lambda r: r.arrival):
            if realtime:
                wait = req.arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
            else:
                req.arrival = 0.0
            req.admitted = time.perf_counter() - t0
            try:
                _solve_one(req, self.ordering, self.mixed, self.restart, self.engine)
            except Exception as exc:
                req.error = repr(exc)
            torch.cuda.synchronize()
            req.finished = time.perf_counter() - t0
        return latency_stats(reqs, t0)
