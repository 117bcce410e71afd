"""Elemental evaluation over buckets of elements of different polynomial degree.

``ElementalBuckets`` keeps every bucket's inputs and outputs resident on the device and runs
the evaluation either as one call of ``hdgx_elemental_buckets`` (the buckets' kernels
concurrently on forked side streams; capturable as one CUDA graph with ``capture()`` /
``replay()``), or degree by degree on one stream (``run_sequential``, the plain per-degree
launches).  Outputs are identical bit for bit either way: every element's arithmetic is the
same, only the launch schedule differs.

``SharedLaunch`` evaluates several independent problems of one element shape (e.g. the
same-degree requests of a serving mix, each with its own physics) as ONE segmented launch
(``hdgx_elemental_shared``), or problem by problem (``run_each``), with identical outputs.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

from ._lib import HdgxElemBucket, check, lib
from .elemental import DArray, DeviceMaster, _require_cuda, _stream_ptr, alloc_elemental_outputs, app_struct


class ElementalBuckets:
    def __init__(self, problem, mixed=False, grids=None):
        """problem: a ``configs.MixedDegreeProblem``; grids: CTAs per bucket (None: one wave)."""
        _require_cuda()
        self.mixed = mixed
        self.buckets = []
        for k, (p, P, idx) in enumerate(problem.buckets):
            sl = np.asarray(idx)
            m = P.mesh
            b = dict(p=p, ne=int(sl.size), master=P.master, app=P.app, dm=DeviceMaster(P.master),
                     appc=app_struct(P.app),
                     dg=DArray.from_numpy(np.asfortranarray(m.dgnodes[..., sl])),
                     bf=DArray.from_numpy(np.asfortranarray(m.bf[:, sl]), dtype=torch.int32),
                     udg=DArray.from_numpy(np.asfortranarray(P.UDG[..., sl])),
                     uh=DArray.from_numpy(np.asfortranarray(P.uh_elem()[..., sl])),
                     sh=DArray.from_numpy(np.asfortranarray(P.SH[..., sl])))
            b["out"] = alloc_elemental_outputs(P.master, P.app, b["ne"])
            self.buckets.append(b)
        self.set_grids(grids)
        self.graph = None

    @property
    def ne(self):
        return sum(b["ne"] for b in self.buckets)

    def set_grids(self, grids):
        self.grids = [0] * len(self.buckets) if grids is None else [int(g) for g in grids]
        arr = (HdgxElemBucket * len(self.buckets))()
        for k, b in enumerate(self.buckets):
            o = b["out"]
            arr[k] = HdgxElemBucket(ct.addressof(b["dm"].c), ct.addressof(b["appc"]), b["ne"], b["dg"].ptr, b["bf"].ptr,
                                    b["udg"].ptr, b["uh"].ptr, b["sh"].ptr, o.AE.ptr, o.FE.ptr, o.DUDG.ptr,
                                    o.DUDG_DUH.ptr, o.status.ptr, self.grids[k])
        self._arr = arr

    def run(self, stream=None):
        """All buckets in one call (concurrent kernels)."""
        rc = lib().hdgx_elemental_buckets(len(self.buckets), ct.cast(self._arr, ct.c_void_p), int(self.mixed),
                                          _stream_ptr(stream))
        check(rc, "hdgx_elemental_buckets")

    def run_sequential(self, stream=None):
        """The plain per-degree launches, one after another on one stream."""
        L = lib()
        fn = L.hdgx_elemental_mixed if self.mixed else L.hdgx_elemental
        for b in self.buckets:
            o = b["out"]
            rc = fn(ct.byref(b["dm"].c), ct.byref(b["appc"]), b["ne"], b["dg"].ptr, b["bf"].ptr, b["udg"].ptr,
                    b["uh"].ptr, b["sh"].ptr, o.AE.ptr, o.FE.ptr, o.DUDG.ptr, o.DUDG_DUH.ptr, o.status.ptr,
                    _stream_ptr(stream))
            check(rc, "hdgx_elemental")

    def capture(self):
        """Capture ``run`` as a CUDA graph (after one uncaptured call, which sets up the side
        streams and shared-memory limits)."""
        self.run()
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run()
        self.graph = g
        return g

    def replay(self):
        self.graph.replay()

    def statuses(self):
        return [int(b["out"].status.numpy().max()) if b["ne"] else 0 for b in self.buckets]


class SharedLaunch:
    """Several problems of one (nd, porder) and one physics kind in one elemental launch."""

    def __init__(self, problems):
        _require_cuda()
        self.items = []
        for P in problems:
            m = P.mesh
            it = dict(P=P, ne=int(m.ne), dm=DeviceMaster(P.master), appc=app_struct(P.app),
                      dg=DArray.from_numpy(m.dgnodes), bf=DArray.from_numpy(m.bf, dtype=torch.int32),
                      udg=DArray.from_numpy(P.UDG), uh=DArray.from_numpy(P.uh_elem()), sh=DArray.from_numpy(P.SH))
            it["out"] = alloc_elemental_outputs(P.master, P.app, it["ne"])
            self.items.append(it)
        arr = (HdgxElemBucket * len(self.items))()
        for k, it in enumerate(self.items):
            o = it["out"]
            arr[k] = HdgxElemBucket(ct.addressof(it["dm"].c), ct.addressof(it["appc"]), it["ne"], it["dg"].ptr,
                                    it["bf"].ptr, it["udg"].ptr, it["uh"].ptr, it["sh"].ptr, o.AE.ptr, o.FE.ptr,
                                    o.DUDG.ptr, o.DUDG_DUH.ptr, o.status.ptr, 0)
        self._arr = arr

    @property
    def ne(self):
        return sum(it["ne"] for it in self.items)

    def run(self, grid=0, stream=None):
        """One launch over every problem's elements (status -2: shapes or physics kinds differ)."""
        rc = lib().hdgx_elemental_shared(len(self.items), ct.cast(self._arr, ct.c_void_p), int(grid),
                                         _stream_ptr(stream))
        check(rc, "hdgx_elemental_shared")

    def run_each(self, stream=None):
        """One hdgx_elemental launch per problem, one after another."""
        L = lib()
        for it in self.items:
            o = it["out"]
            rc = L.hdgx_elemental(ct.byref(it["dm"].c), ct.byref(it["appc"]), it["ne"], it["dg"].ptr, it["bf"].ptr,
                                  it["udg"].ptr, it["uh"].ptr, it["sh"].ptr, o.AE.ptr, o.FE.ptr, o.DUDG.ptr,
                                  o.DUDG_DUH.ptr, o.status.ptr, _stream_ptr(stream))
            check(rc, "hdgx_elemental")

    def outputs(self):
        return [[getattr(it["out"], k).numpy().copy() for k in ("AE", "FE", "DUDG", "DUDG_DUH", "status")]
                for it in self.items]
