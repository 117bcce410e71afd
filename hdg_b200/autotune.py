"""Launch-schedule autotuner for the bucketed elemental evaluation.

For every bucket (one polynomial degree) the elemental kernel's shared-memory plan and tile
width are fixed at compile time by the degree; what is left to choose at run time is the
schedule: how many CTAs each bucket's launch gets when the buckets run concurrently, and
whether concurrency pays at all.  ``tune_buckets`` times, as CUDA-graph replays, (a) one
resident wave per bucket, (b) grids proportional to each bucket's measured solo time (the SMs
shared out so that the buckets finish together), (c) the plain per-degree launches one after
another, and keeps the fastest.  Every candidate computes identical outputs.
"""
from __future__ import annotations

import torch


def _time(fn, reps):
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fn()
    torch.cuda.synchronize()
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def resident_wave(per_sm=2):
    return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count * per_sm


def tune_buckets(eb, reps=3):
    """Returns (best schedule name, grids, {name: ms}) and leaves ``eb`` set to the best."""
    nb = len(eb.buckets)
    wave = resident_wave()
    # solo time of every bucket (one wave, alone on the GPU)
    solo = []
    for k in range(nb):
        grids = [0] * nb
        eb.set_grids(grids)
        sub = eb._arr
        import ctypes as ct
        from ._lib import check, lib
        from .elemental import _stream_ptr

        def one(k=k):
            check(lib().hdgx_elemental_buckets(1, ct.byref(sub[k]), int(eb.mixed), _stream_ptr(None)), "buckets")
        solo.append(_time(one, reps))
    tot = sum(solo)
    prop = [max(1, int(round(wave * s / tot))) for s in solo]
    results = {}
    for name, grids in (("wave_per_bucket", [0] * nb), ("proportional", prop)):
        eb.set_grids(grids)
        eb.capture()
        results[name] = _time(eb.replay, reps)
    results["per_degree_sequential"] = _time(eb.run_sequential, reps)
    best = min(results, key=results.get)
    grids = {"wave_per_bucket": [0] * nb, "proportional": prop}.get(best, [0] * nb)
    eb.set_grids(grids)
    eb.graph = None
    return best, grids, results, solo
