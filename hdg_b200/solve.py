"""Newton solve of a steady HDG problem on the GPU (the reference's hdg_solve call surface).

``hdg_solve(master, mesh, app, UDG, UH, SH)`` follows kernel/hdg_solve.m:104-176:
  assemble (elemental kernel + block-CSR global assembly) -> F, K, DUDG, DUDG_DUH
  while |F|/|F0| > tol and it < maxiter:
      DUH   = K \\ F           (BILU(0)-preconditioned GMRES on the GPU; the reference's
                               default is a sparse direct K\\F, hdg_solve.m:111)
      DUDGT = DUDG + DUDG_DUH DUH(elcon)                      (hdg_solve.m:119-121)
      damped update UDG += alfa DUDGT, UH += alfa DUH with alfa halved while |F| grows
      (hdg_solve.m:139-163)
Everything stays resident on the device across iterations; only scalars come back.
"""
from __future__ import annotations

import ctypes as ct
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from ._lib import HdgxAssemblyMap, HdgxBsr, check, lib
from .elemental import (DArray, DeviceMaster, alloc_elemental_outputs, app_struct, as_darray, getq, _require_cuda,
                        _stream_ptr, stored_components)
from .ordering import assembly_map, levels_of_order, multicolor, sweep_plan


class TraceSystem:
    """Device-resident block-CSR pattern, elimination order and assembly map of a mesh."""

    def __init__(self, mesh, master, app, ordering=None):
        """ordering: "mdf" (default; the reference's minimum-discarded-fill order, computed from
        the first assembled matrix, eliminated with flag-synchronised sweeps), "multicolor"
        (greedy colouring, one launch per colour), or an ``Ordering``."""
        _require_cuda()
        self.nf, self.npf, self.nfe, self.ncu = mesh.nf, master.npf, master.nfe, app.ncu
        self.bs = app.ncu * master.npf
        self.nnzb = int(mesh.cbsr_rowpts[-1])
        self.rowpts_h = np.ascontiguousarray(mesh.cbsr_rowpts, dtype=np.int64)
        self.colind_h = np.ascontiguousarray(mesh.cbsr_colind, dtype=np.int32)
        ordering = "mdf" if ordering is None else ordering
        self.pending_mdf = isinstance(ordering, str) and ordering == "mdf"
        if isinstance(ordering, str):
            self.ord = multicolor(mesh.cbsr_rowpts, mesh.cbsr_colind, mesh.nf)
        else:
            self.ord = ordering
        am = assembly_map(mesh.t2f, mesh.cbsr_rowpts, mesh.cbsr_colind)
        i32 = torch.int32
        self.d = dict(
            rowpts=DArray.from_numpy(np.asarray(mesh.cbsr_rowpts, dtype=np.int64), dtype=torch.int64),
            colind=DArray.from_numpy(mesh.cbsr_colind, dtype=i32),
            color_rows=DArray.from_numpy(self.ord.color_rows, dtype=i32),
            pos=DArray.from_numpy(self.ord.pos, dtype=i32),
            blk_e=DArray.from_numpy(am.blk_e, dtype=i32), blk_ab=DArray.from_numpy(am.blk_ab, dtype=i32),
            blk_row=DArray.from_numpy(am.blk_row, dtype=i32), face_e=DArray.from_numpy(am.face_e, dtype=i32),
            face_a=DArray.from_numpy(am.face_a, dtype=i32), elcon=DArray.from_numpy(mesh.elcon, dtype=i32))
        self.color_ptr = np.ascontiguousarray(self.ord.color_ptr, dtype=np.int32)
        self.sched = torch.zeros(4 + self.nf, dtype=torch.int32, device="cuda")
        d = self.d
        d["color_ptr"] = DArray.from_numpy(self.color_ptr, dtype=torch.int32)
        self.bsr = HdgxBsr(self.nf, self.bs, self.nnzb, d["rowpts"].ptr, d["colind"].ptr, self.ord.ncolors,
                           self.color_ptr.ctypes.data, d["color_rows"].ptr, d["pos"].ptr, None)
        self.map = HdgxAssemblyMap(d["blk_e"].ptr, d["blk_ab"].ptr, d["blk_row"].ptr, d["face_e"].ptr,
                                   d["face_a"].ptr)

    def set_levels(self, o2u, u2o):
        """Eliminate in the sequential order o2u, level by level (one launch per level)."""
        self.o2u = np.ascontiguousarray(o2u, dtype=np.int32)
        self.u2o = np.ascontiguousarray(u2o, dtype=np.int32)
        lv = levels_of_order(self.rowpts_h, self.colind_h, self.o2u, self.u2o)
        self.ord = lv
        self.d["color_rows"] = DArray.from_numpy(lv.color_rows, dtype=torch.int32)
        self.d["pos"] = DArray.from_numpy(lv.pos, dtype=torch.int32)
        self.color_ptr = np.ascontiguousarray(lv.color_ptr, dtype=np.int32)
        self.d["color_ptr"] = DArray.from_numpy(self.color_ptr, dtype=torch.int32)
        self.bsr.ncolors = lv.ncolors
        self.bsr.color_ptr = self.color_ptr.ctypes.data
        self.bsr.color_rows = self.d["color_rows"].ptr
        self.bsr.pos = self.d["pos"].ptr
        self.bsr.sched = None
        plan, maxd = sweep_plan(lv, self.rowpts_h, self.colind_h)
        if plan is not None:
            self.d["sweep_plan"] = DArray.from_numpy(plan, dtype=torch.int32)
            self.bsr.sweep_plan = self.d["sweep_plan"].ptr
            self.bsr.sweep_maxd = maxd
        self.pending_mdf = False

    def set_order(self, o2u, u2o):
        """Eliminate rows one after another in the order o2u (flag-synchronised sweeps)."""
        self.o2u = np.ascontiguousarray(o2u, dtype=np.int32)
        self.u2o = np.ascontiguousarray(u2o, dtype=np.int32)
        self.d["color_rows"] = DArray.from_numpy(self.o2u, dtype=torch.int32)
        self.d["pos"] = DArray.from_numpy(self.u2o, dtype=torch.int32)
        self.color_ptr = np.array([0, self.nf], dtype=np.int32)
        self.sched.zero_()
        self.bsr.ncolors = 0
        self.bsr.color_ptr = self.color_ptr.ctypes.data
        self.bsr.color_rows = self.d["color_rows"].ptr
        self.bsr.pos = self.d["pos"].ptr
        self.bsr.sched = self.sched.data_ptr()
        self.bsr.sweep_plan = None
        self.pending_mdf = False

    def mdf_order(self, Hg, stream=None):
        """computeMDFordering.m: block norms on the GPU, greedy selection on the host."""
        C = torch.empty(self.nnzb, dtype=torch.float64, device="cuda")
        check(lib().hdgx_block_norms(ct.byref(self.bsr), Hg.ptr, C.data_ptr(), _stream_ptr(stream)), "hdgx_block_norms")
        Ch = np.ascontiguousarray(C.cpu().numpy())
        o2u = np.zeros(self.nf, dtype=np.int32)
        u2o = np.zeros(self.nf, dtype=np.int32)
        rc = lib().hdgx_mdf_ordering(self.nf, self.rowpts_h.ctypes.data, self.colind_h.ctypes.data, Ch.ctypes.data,
                                     o2u.ctypes.data, u2o.ctypes.data)
        check(rc, "hdgx_mdf_ordering")
        return o2u, u2o

    def empty_blocks(self):
        return DArray.empty((self.bs, self.bs, self.nnzb))

    def empty_vec(self):
        return DArray.empty((self.bs, self.nf))

    # ------------------------------------------------------------ operations
    def assemble(self, AE, FE, Hg, Rg, stream=None):
        rc = lib().hdgx_globalassembly(ct.byref(self.bsr), ct.byref(self.map), self.ncu, self.npf, self.nfe,
                                       self.d["elcon"].ptr, AE.ptr, FE.ptr, Hg.ptr, Rg.ptr, _stream_ptr(stream))
        check(rc, "hdgx_globalassembly")

    def matvec(self, Hg, x, y, stream=None):
        check(lib().hdgx_matvec(ct.byref(self.bsr), Hg.ptr, x.ptr, y.ptr, _stream_ptr(stream)), "hdgx_matvec")

    def bilu0(self, Hg, Mg, status=None, stream=None):
        if self.pending_mdf:
            self.set_levels(*self.mdf_order(Hg, stream))
        Mg.t.copy_(Hg.t)
        st = status.ptr if status is not None else None
        check(lib().hdgx_bilu0_factor(ct.byref(self.bsr), Mg.ptr, st, _stream_ptr(stream)), "hdgx_bilu0_factor")

    def bilu0_apply(self, Mg, x, v, work, stream=None):
        check(lib().hdgx_bilu0_apply(ct.byref(self.bsr), Mg.ptr, x.ptr, v.ptr, work.ptr, _stream_ptr(stream)),
              "hdgx_bilu0_apply")

    def gmres(self, Hg, Mg, b, x, restart=20, tol=1e-10, maxit=1000, workspace=None, stream=None):
        it, fl, rr = ct.c_int(0), ct.c_int(0), ct.c_double(0.0)
        hist = np.zeros(maxit + 1)
        ws = workspace.data_ptr() if workspace is not None else None
        rc = lib().hdgx_gmres_bilu0(ct.byref(self.bsr), Hg.ptr, Mg.ptr, b.ptr, x.ptr, int(restart), float(tol),
                                    int(maxit), ct.byref(it), ct.byref(fl), ct.byref(rr),
                                    hist.ctypes.data_as(ct.c_void_p), ws, _stream_ptr(stream))
        check(rc, "hdgx_gmres_bilu0")
        return it.value, fl.value, rr.value, hist[:it.value]

    def gmres_mixed(self, Hg, Mg, Mg32, b, x, restart=20, tol=1e-10, maxit=1000, workspace=None, stream=None):
        """gmres with the factors Mg converted to FP32 (Mg32, a float32 tensor of Mg's size) and
        read in FP32 by the level sweeps; the rest of GMRES stays FP64."""
        st = _stream_ptr(stream)
        check(lib().hdgx_bilu0_to_f32(ct.byref(self.bsr), Mg.ptr, Mg32.data_ptr(), st), "hdgx_bilu0_to_f32")
        it, fl, rr = ct.c_int(0), ct.c_int(0), ct.c_double(0.0)
        hist = np.zeros(maxit + 1)
        ws = workspace.data_ptr() if workspace is not None else None
        rc = lib().hdgx_gmres_bilu0_mixed(ct.byref(self.bsr), Hg.ptr, Mg32.data_ptr(), b.ptr, x.ptr, int(restart),
                                          float(tol), int(maxit), ct.byref(it), ct.byref(fl), ct.byref(rr),
                                          hist.ctypes.data_as(ct.c_void_p), ws, st)
        check(rc, "hdgx_gmres_bilu0_mixed")
        return it.value, fl.value, rr.value, hist[:it.value]

    def workspace(self, restart):
        nb = lib().hdgx_gmres_workspace_bytes(ct.byref(self.bsr), int(restart))
        return torch.empty(int(nb), dtype=torch.uint8, device="cuda")


@dataclass
class SolveReport:
    iterations: int = 0
    residuals: list = field(default_factory=list)       # |F| after every Newton step (F0 first)
    alphas: list = field(default_factory=list)
    gmres_iters: list = field(default_factory=list)
    gmres_relres: list = field(default_factory=list)
    times: dict = field(default_factory=dict)
    converged: bool = False


class HDGSolver:
    """Device-resident state of one steady problem (mesh, master, app) for Newton steps."""

    def __init__(self, master, mesh, app, ordering=None, restart=20, mixed=False, denseblock=False):
        """denseblock=True solves each Newton step's linear system as the reference does with
        app.denseblock = 1: mkDenseBlockSystem.m's scaled face blocks and gmres.m (no BILU(0))."""
        _require_cuda()
        self.master, self.mesh, self.app = master, mesh, app
        self.mixed = mixed
        self.dm = DeviceMaster(master)
        self.ts = TraceSystem(mesh, master, app, ordering)
        ne = mesh.ne
        self.ne = ne
        self.dg = DArray.from_numpy(mesh.dgnodes)
        self.bf = DArray.from_numpy(mesh.bf, dtype=torch.int32)
        self.out = alloc_elemental_outputs(master, app, ne)
        self.Hg = self.ts.empty_blocks()
        self.Mg = self.ts.empty_blocks()
        self.Rg = self.ts.empty_vec()
        self.DUH = self.ts.empty_vec()
        self.work = self.ts.empty_vec()
        ndf = master.npf * master.nfe
        self.UHe = DArray.empty((app.ncu, ndf, ne))
        self.nco = stored_components(app)             # nc, or ncu when app.getdqdg = 0
        self.DUDGT = DArray.empty((master.npv, self.nco, ne))
        self.app_c = app_struct(app)
        self.restart = restart
        self.denseblock = denseblock
        if denseblock:
            from .dense import DenseBlockSystem
            self.dense = DenseBlockSystem(self.ts, mesh)
            self.ws = None
        else:
            self.ws = self.ts.workspace(restart)

    def gather(self, UH, stream=None):
        ndf = self.master.npf * self.master.nfe
        check(lib().hdgx_gather_uh(self.app.ncu, ndf, self.ne, self.ts.d["elcon"].ptr, UH.ptr, self.UHe.ptr,
                                   _stream_ptr(stream)), "hdgx_gather_uh")

    def assemble(self, UDG, UH, SH, stream=None):
        """hdg_assemble: elemental kernel + global assembly; returns |F|."""
        self.gather(UH, stream)
        L = lib()
        o = self.out
        fn = L.hdgx_elemental_mixed if self.mixed else L.hdgx_elemental
        rc = fn(ct.byref(self.dm.c), ct.byref(self.app_c), self.ne, self.dg.ptr, self.bf.ptr, UDG.ptr,
                self.UHe.ptr, SH.ptr, o.AE.ptr, o.FE.ptr, o.DUDG.ptr, o.DUDG_DUH.ptr, o.status.ptr,
                _stream_ptr(stream))
        check(rc, "hdgx_elemental")
        self.ts.assemble(o.AE, o.FE, self.Hg, self.Rg, stream)
        return float(torch.linalg.vector_norm(self.Rg.t).item())

    def linear_solve(self, tol=1e-10, maxit=1000, stream=None):
        """DUH = K \\ F with BILU(0)-GMRES, or with the dense face-block GMRES (x0 = 0)."""
        self.DUH.t.zero_()
        if self.denseblock:
            self.dense.build(self.Hg, self.Rg, stream)
            return self.dense.gmres(self.DUH, restart=self.restart, tol=tol, maxit=maxit, stream=stream)
        self.ts.bilu0(self.Hg, self.Mg, stream=stream)
        if self.mixed and self.ts.bsr.sweep_plan:
            # mixed precision: the preconditioner's factors read in FP32 by the level sweeps
            if getattr(self, "Mg32", None) is None:
                self.Mg32 = torch.empty(self.Mg.t.numel(), dtype=torch.float32, device=self.Mg.t.device)
            return self.ts.gmres_mixed(self.Hg, self.Mg, self.Mg32, self.Rg, self.DUH, self.restart, tol, maxit,
                                       self.ws, stream)
        return self.ts.gmres(self.Hg, self.Mg, self.Rg, self.DUH, self.restart, tol, maxit, self.ws, stream)

    def backsub(self, stream=None):
        m, a = self.master, self.app
        ndf = m.npf * m.nfe
        o = self.out
        check(lib().hdgx_backsub(m.npv, self.nco, a.ncu, ndf, self.ne, self.ts.d["elcon"].ptr, o.DUDG.ptr,
                                 o.DUDG_DUH.ptr, self.DUH.ptr, self.DUDGT.ptr, _stream_ptr(stream)), "hdgx_backsub")

    def update(self, UDG, UH, UDG0, UH0, alfa, SH):
        """UDG(:,1:nco,:) = UDG0 + alfa DUDGT, UH = UH0 + alfa DUH (hdg_solve.m:145-146); with
        app.getdqdg = 0 the q part is then recovered with getq (hdg_solve.m:148-151)."""
        if self.nco == self.app.nc:
            torch.add(UDG0, self.DUDGT.t, alpha=alfa, out=UDG.t)
        else:
            ne, npv, nc, nco = self.ne, self.master.npv, self.app.nc, self.nco
            u = UDG.t.view(ne, nc, npv)
            u.copy_(UDG0.view(ne, nc, npv))
            u[:, :nco, :].add_(self.DUDGT.t.view(ne, nco, npv), alpha=alfa)
        torch.add(UH0, self.DUH.t.view(-1), alpha=alfa, out=UH.t)
        if self.nco != self.app.nc:
            self.gather(UH)
            Q, _ = getq(self.master, self.app, self.dg, self.bf, UDG, self.UHe, SH, dmaster=self.dm)
            ne, npv, nc, ncu = self.ne, self.master.npv, self.app.nc, self.app.ncu
            UDG.t.view(ne, nc, npv)[:, ncu:, :].copy_(Q.t.view(ne, nc - ncu, npv))

    def solve(self, UDG, UH, SH, tol=1e-10, maxiter=16, gmres_tol=1e-10, gmres_maxit=1000, linear=False):
        """The Newton loop of hdg_solve.m; UDG [npv,nc,ne], UH [ncu,nsiz] device arrays (updated)."""
        rep = SolveReport()
        t0 = time.perf_counter()
        F = self.assemble(UDG, UH, SH)
        F0 = F
        rep.residuals.append(F)
        rel = 1.0
        it = 0
        UDG0 = torch.empty_like(UDG.t)
        UH0 = torch.empty_like(UH.t)
        while rel > tol and it < maxiter:
            gi, gf, grr, _ = self.linear_solve(gmres_tol, gmres_maxit)
            rep.gmres_iters.append(gi)
            rep.gmres_relres.append(grr)
            self.backsub()
            if linear:
                UDG0.copy_(UDG.t)
                UH0.copy_(UH.t)
                self.update(UDG, UH, UDG0, UH0, 1.0, SH)
                rep.iterations = 1
                return rep
            it += 1
            UDG0.copy_(UDG.t)
            UH0.copy_(UH.t)
            duh0 = F
            alfa = 1.0
            while True:
                self.update(UDG, UH, UDG0, UH0, alfa, SH)
                F = self.assemble(UDG, UH, SH)
                if F > duh0:
                    alfa /= 2
                    if alfa < 1e-2:
                        break
                else:
                    break
            rep.alphas.append(alfa)
            rep.residuals.append(F)
            rel = F / F0 if F0 > 0 else 0.0
        torch.cuda.synchronize()
        rep.iterations = it
        rep.converged = rel <= tol
        rep.times["total_s"] = time.perf_counter() - t0
        return rep


def hdg_solve(master, mesh, app, UDG, UH, SH=None, tol=1e-10, maxiter=16, gmres_tol=1e-10, restart=20,
              ordering=None, mixed=False, denseblock=None):
    """kernel/hdg_solve.m: returns (UDG, UH, report) as host arrays (inputs are not modified).
    ``mixed=True`` assembles with the mixed-precision elemental kernel; ``denseblock`` (default
    ``app.denseblock`` when the app has it) selects the dense face-block GMRES of
    hdg_solve.m:88-92,110-116 instead of BILU(0)-GMRES."""
    if denseblock is None:
        denseblock = bool(getattr(app, "denseblock", 0))
    s = HDGSolver(master, mesh, app, ordering=ordering, restart=restart, mixed=mixed, denseblock=denseblock)
    dU = DArray.from_numpy(UDG)
    dH = DArray.from_numpy(UH)
    SH = np.zeros_like(UDG) if SH is None else np.array(SH, dtype=np.float64, copy=True)
    SH[:, app.ncu:, :] = 0.0                     # hdg_solve.m:62-63 (no wave formulation here)
    dS = DArray.from_numpy(SH)
    rep = s.solve(dU, dH, dS, tol=tol, maxiter=maxiter, gmres_tol=gmres_tol)
    return dU.numpy(), dH.numpy(), rep


class Combiner:
    """Shared elemental launches of concurrent native solves (``hdgx_combiner`` of the C ABI).

    Solves that pass the same combiner to ``hdgx_solve`` and run at the same time (each on its
    own thread and CUDA stream) have their assemblies' elemental evaluations batched: every group
    of equal master tables and one physics kind runs as one ``hdgx_elemental_shared`` launch.
    ``window_us``: how long the first assembly of a batch waits for the other attached solves
    (0: it takes what is queued at once)."""

    def __init__(self, window_us=0):
        _require_cuda()
        h = ct.c_void_p()
        check(lib().hdgx_combiner_create(int(window_us), ct.byref(h)), "hdgx_combiner_create")
        self.handle = h
        self.window_us = int(window_us)

    def stats(self):
        b, n, s = ct.c_longlong(), ct.c_longlong(), ct.c_longlong()
        check(lib().hdgx_combiner_stats(self.handle, ct.byref(b), ct.byref(n), ct.byref(s)), "hdgx_combiner_stats")
        k, w = ct.c_double(), ct.c_double()
        check(lib().hdgx_combiner_times(self.handle, ct.byref(k), ct.byref(w)), "hdgx_combiner_times")
        return {"batches": b.value, "launches": n.value, "submissions": s.value, "key_s": k.value,
                "submit_s": w.value}

    def close(self):
        if self.handle:
            check(lib().hdgx_combiner_destroy(self.handle), "hdgx_combiner_destroy")
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def hdgx_solve(master, mesh, app, UDG, UH, SH=None, tol=1e-10, maxiter=16, gmres_tol=1e-10, restart=20,
               ordering="mdf", mixed=False, gmres_maxit=1000, stream=None, combiner=None):
    """kernel/hdg_solve.m as ONE native call (``hdgx_solve`` of the C ABI): the Newton loop,
    the elimination order and the assembly map are built inside the library.  Returns
    (UDG, UH, report dict) as host arrays; the inputs are not modified.  ``combiner``: a
    ``Combiner`` shared with concurrent solves (``hdgx_solve_combined``, FP64 only)."""
    from ._lib import HDGX_SOLVE_MAXIT, HdgxMesh, HdgxSolveOpts, HdgxSolveReport
    _require_cuda()
    if maxiter > HDGX_SOLVE_MAXIT:
        raise ValueError(f"maxiter <= {HDGX_SOLVE_MAXIT}")
    dm = DeviceMaster(master)
    appc = app_struct(app)
    dg = DArray.from_numpy(mesh.dgnodes)
    bf = DArray.from_numpy(mesh.bf, dtype=torch.int32)
    el = DArray.from_numpy(mesh.elcon, dtype=torch.int32)
    t2f = np.asfortranarray(mesh.t2f, dtype=np.int32)
    rp = np.ascontiguousarray(mesh.cbsr_rowpts, dtype=np.int64)
    ci = np.ascontiguousarray(mesh.cbsr_colind, dtype=np.int32)
    cm = HdgxMesh(mesh.ne, mesh.nf, dg.ptr, bf.ptr, el.ptr, t2f.ctypes.data, rp.ctypes.data, ci.ctypes.data)
    opts = HdgxSolveOpts({"mdf": 0, "multicolor": 1}[ordering], int(mixed), int(restart), int(maxiter), float(tol),
                         float(gmres_tol), int(gmres_maxit))
    dU = DArray.from_numpy(UDG)
    dH = DArray.from_numpy(UH)
    dS = DArray.from_numpy(np.zeros_like(UDG) if SH is None else SH)
    rep = HdgxSolveReport()
    if combiner is None:
        rc = lib().hdgx_solve(ct.byref(dm.c), ct.byref(appc), ct.byref(cm), dU.ptr, dH.ptr, dS.ptr, ct.byref(opts),
                              ct.byref(rep), _stream_ptr(stream))
    else:
        rc = lib().hdgx_solve_combined(ct.byref(dm.c), ct.byref(appc), ct.byref(cm), dU.ptr, dH.ptr, dS.ptr,
                                       ct.byref(opts), ct.byref(rep), combiner.handle, _stream_ptr(stream))
    check(rc, "hdgx_solve")
    n = rep.iterations
    report = dict(iterations=n, converged=bool(rep.converged), levels=rep.ncolors,
                  residuals=list(rep.residuals[:n + 1]), alphas=list(rep.alphas[:n]),
                  gmres_iters=list(rep.gmres_iters[:n]), gmres_relres=list(rep.gmres_relres[:n]),
                  graph_assemblies=rep.graph_assemblies)
    return dU.numpy(), dH.numpy(), report
