#!/usr/bin/env python
"""Benchmark of the HDG elemental step on B200.

One step = one fused FP64 elemental evaluation (volume + face integrals + local (u,q) Schur
elimination -> AE, FE, DUDG, DUDG_DUH) over every element of the workload, inputs resident
in HBM.  Workload (the FP64-vs-mixed Navier-Stokes configuration): 2D steady compressible
Navier-Stokes, Re 1000, Pr 0.72, Mach 0.3, [0,1]^2 as 128x128 squares x 2 triangles =
32,768 elements, p = 3 (local (u,q) block 120x120, trace block 48x48), seeded synthetic state.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config c2]

Under torchrun each rank evaluates its own copy of the mesh (elements are independent: weak
scaling, no data-path collective); value = elements of all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np
import psutil

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "HDG elem Schur-solves/s (mixed vs FP64, rel err≤1e-10); serve solves/s, p50/p99"
UNIT = "elements/s"

WORKLOADS = {
    "c2": dict(name="c2", kw=dict(n=128, porder=3),
               desc="2D steady Navier-Stokes Re=1000 Pr=0.72 M=0.3, [0,1]^2 128x128x2 = 32768 triangles, p=3"),
    "c1": dict(name="c1", kw=dict(n=16, porder=2),
               desc="2D steady Euler M=0.5 + vortex, [0,10]^2 16x16x2 = 512 triangles, p=2"),
    "c4": dict(name="c4", kw=dict(n=32, porder=2),
               desc="3D steady Euler M=0.4, unit cube 32^3x6 = 196608 tets, p=2"),
}


def max_over_ranks(ms, ws, device):
    """The slowest rank's time (every rank takes part; world size 1: unchanged)."""
    if ws <= 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, ws, steps, total_ms):
    """Whole-job throughput: the units of all ranks over the slowest rank's time."""
    return ws * units_per_rank * steps / (total_ms * 1e-3)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi samples (every 200 ms) of SM clock and throttle reasons during a region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def measure_fp64_peak(torch):
    """cuBLAS DGEMM throughput (TFLOP/s) on this GPU, the FP64 roofline denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(4):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return json.loads(p.read_text()), "measured"
        except ValueError:
            pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def profile_traffic(kernel_tag, variant):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of this kernel
    variant from its committed ncu summary, if any."""
    f = ROOT / "profiles" / f"{kernel_tag}.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.strip().startswith(f"dram_bytes_per_launch_{variant}:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


def cpu_baseline(P, nsample, nthreads):
    """The CPU oracle (C restatement of the reference path) on a bounded element sample."""
    from oracle import oracle as O
    sl = slice(0, min(nsample, P.mesh.ne))
    args = (P.master, P.app, np.asfortranarray(P.mesh.dgnodes[..., sl]), np.asfortranarray(P.mesh.bf[:, sl]),
            np.asfortranarray(P.UDG[..., sl]), np.asfortranarray(P.uh_elem()[..., sl]),
            np.asfortranarray(P.SH[..., sl]))
    O.hdg_elemental(*args[:2], *[a[..., :8] if a.ndim > 1 else a for a in args[2:]], nthreads=nthreads)
    t0 = time.perf_counter()
    O.hdg_elemental(*args, nthreads=nthreads)
    dt = time.perf_counter() - t0
    n = sl.stop - sl.start
    return n / dt, n, dt


def cpu_baseline_timed(P, nthreads, seconds):
    """The CPU oracle over the whole workload, repeated until about ``seconds`` have passed."""
    v, n, dt = cpu_baseline(P, P.mesh.ne, nthreads)
    tot_n, tot_t = n, dt
    while tot_t < seconds:
        v, n, dt = cpu_baseline(P, P.mesh.ne, nthreads)
        tot_n += n
        tot_t += dt
    return tot_n / tot_t, tot_n, tot_t


def cpu_reference_schur(P, nsample=2048):
    """The reference's own local Schur MEX, kernel/schur_uq.c (compiled from the reference tree
    into oracle/_ref with the project's MEX emulation), on the blocks M, C, E, BD, F, GK, H, Rq,
    Ru, Rh that the oracle's volint/faceint produce for the first ``nsample`` elements: once as
    the reference runs it (its serial element loop, schur_uq.c:263-287, on one core), and once
    with the element range split across all host cores (one MEX call per core on its share)."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    if not O.ref_available():
        return {"unavailable": "the reference's schur_uq.c was not compiled into oracle/_ref"}
    n = min(nsample, P.mesh.ne)
    sl = slice(0, n)
    nth = os.cpu_count() or 1
    blk = O.hdg_elemental(P.master, P.app, np.asfortranarray(P.mesh.dgnodes[..., sl]),
                          np.asfortranarray(P.mesh.bf[:, sl]), np.asfortranarray(P.UDG[..., sl]),
                          np.asfortranarray(P.uh_elem()[..., sl]), np.asfortranarray(P.SH[..., sl]),
                          intermediates=True, nthreads=nth)
    keys = ("M", "C", "E", "BD", "F", "GK", "H", "Rq", "Ru", "Rh")
    npv, ncu, nc = P.master.npv, P.app.ncu, P.app.nc
    ndf = P.master.npf * P.master.nfe

    def prepared(a, b):
        shapes = [(npv, nc, b - a), (npv, nc, ncu, ndf, b - a), (ncu, ndf, ncu, ndf, b - a), (ncu, ndf, b - a)]
        return O.ref_mex_call("schur_uq.so", [np.asfortranarray(blk[k][..., a:b]) for k in keys], shapes)

    run, outs = prepared(0, n)
    t0 = time.perf_counter()
    run()
    t_serial = time.perf_counter() - t0
    err = float(np.abs(outs[3] - blk["FE"]).max() / np.abs(blk["FE"]).max())   # the MEX's FE vs the oracle's
    cuts = np.linspace(0, n, nth + 1).astype(int)
    calls = [prepared(a, b)[0] for a, b in zip(cuts[:-1], cuts[1:]) if b > a]
    with ThreadPoolExecutor(len(calls)) as ex:              # ctypes releases the GIL in the MEX
        t0 = time.perf_counter()
        list(ex.map(lambda f: f(), calls))
        t_par = time.perf_counter() - t0
    return {"code": "kernel/schur_uq.c (reference source, unmodified) via oracle/_ref/schur_uq.so",
            "sample": f"{n} elements of the workload (blocks from the oracle's volint/faceint)",
            "serial": {"value": n / t_serial, "unit": UNIT, "cores": 1, "s": t_serial},
            "all_cores": {"value": n / t_par, "unit": UNIT, "cores": len(calls), "s": t_par},
            "FE_rel_diff_vs_oracle": err}


def cpu_newton_step(P, gpu_gmres_iters, gmres_sample=20):
    """One Newton iteration of kernel/hdg_solve.m:104-176 with the CPU oracle (assembly on all
    host threads; MDF order, BILU(0) factor, GMRES and back-substitution in its single-threaded
    C): the assembly, MDF order, factor, back-substitution and line-search re-assembly are timed
    in full; GMRES is timed over ``gmres_sample`` iterations and scaled to the iteration count
    the same step takes on the GPU (the oracle's MDF-ordered GMRES takes the same count)."""
    from oracle import oracle as O
    from hdg_b200.app import gather_uh
    m, a, mesh = P.master, P.app, P.mesh
    nth = os.cpu_count() or 1
    SH = np.array(P.SH, order="F", copy=True)
    SH[:, a.ncu:, :] = 0.0
    t = {}
    t0 = time.perf_counter()
    r = O.hdg_elemental(m, a, mesh.dgnodes, mesh.bf, P.UDG, gather_uh(P.UH, mesh.elcon), SH, nthreads=nth)
    Hg, Rg = O.globalassembly(mesh, r["AE"], r["FE"], m.npf, a.ncu)
    t["assemble_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    o2u, u2o = O.mdf_ordering(mesh, Hg)
    t["mdf_order_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    Mg, _ = O.bilu0(mesh, Hg, o2u, u2o)
    t["bilu0_factor_s"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    DUH, _, it, _ = O.gmres_bilu0(mesh, Mg, Hg, Rg, np.zeros_like(Rg), o2u, u2o, 20, 1e-10, gmres_sample)
    t_g = time.perf_counter() - t0
    t["gmres_s_per_iteration"] = t_g / max(it, 1)
    t0 = time.perf_counter()
    O.backsub(mesh, r["DUDG"], r["DUDG_DUH"], DUH.reshape(a.ncu, mesh.nsiz, order="F"))
    t["backsub_s"] = time.perf_counter() - t0
    est = 2 * t["assemble_s"] + t["mdf_order_s"] + t["bilu0_factor_s"] + t["backsub_s"] + \
        t["gmres_s_per_iteration"] * gpu_gmres_iters
    return {"value": mesh.ne / est, "unit": UNIT, "s": est, "cores_assembly": nth, "cores_linear_solve": 1,
            "kind": "port", "sample": f"assembly x2 (the step and its line-search re-assembly), MDF order, factor and "
                                       f"back-substitution timed in full; GMRES timed over {it} iterations and scaled "
                                       f"to {gpu_gmres_iters}", "parts": t}


def run_reference(args, wl):
    """--impl reference: the reference path's CPU implementation on the host cores."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from hdg_b200 import configs
    P = configs.by_name(wl["name"], **wl["kw"])
    nthreads = os.cpu_count() or 1
    nsample = P.mesh.ne                     # every step evaluates every element of the workload
    for _ in range(args.warmup):
        cpu_baseline(P, min(nsample, 512), nthreads)
    vals = []
    t_all = 0.0
    for _ in range(args.steps):
        v, n, dt = cpu_baseline(P, nsample, nthreads)
        vals.append(v)
        t_all += dt
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * P.mesh.ne / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded PCG64 state on a generated mesh)",
        "config": {"workload": wl["desc"], "step": "hdg_elemental over all elements"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                         "sample": f"all {nsample} elements per step, C oracle (volint+faceint+schur_uq2 restated from the reference) on {nthreads} threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-newton", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--no-buckets", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["mixed", "fp64"])
    ap.add_argument("--n", type=int, default=None, help="squares/cubes per side (smaller profiling cases)")
    ap.add_argument("--porder", type=int, default=None, help="polynomial degree (another bucket of the workload)")
    ap.add_argument("--serve-c5", type=int, default=0, metavar="N",
                    help="only the serving measurement on N requests of the full C5 distribution (n 24-180)")
    args = ap.parse_args()
    if args.serve_c5 > 0:
        import torch
        print(json.dumps(serve_c5(torch, args.serve_c5)), flush=True)
        return 0
    wl = dict(WORKLOADS[args.config])
    if args.n is not None:
        wl["kw"] = dict(wl["kw"], n=args.n)
        wl["desc"] = wl["desc"] + f" [reduced: n={args.n} per side]"
    if args.porder is not None:
        wl["kw"] = dict(wl["kw"], porder=args.porder)
        wl["desc"] = wl["desc"].rsplit("p=", 1)[0] + f"p={args.porder}" + (f" [reduced: n={args.n} per side]" if args.n else "")
    if args.impl == "reference":
        return run_reference(args, wl)

    import torch
    import torch.distributed as dist
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from hdg_b200 import configs
    from hdg_b200.elemental import DArray, DeviceMaster, alloc_elemental_outputs, hdg_elemental
    from hdg_b200.perfmodel import element_counts

    P = configs.by_name(wl["name"], seed=rank, **wl["kw"])
    m, a = P.master, P.app
    ne = P.mesh.ne
    dm = DeviceMaster(m)
    d_in = dict(dg=DArray.from_numpy(P.mesh.dgnodes), bf=DArray.from_numpy(P.mesh.bf, dtype=torch.int32),
                udg=DArray.from_numpy(P.UDG), uh=DArray.from_numpy(P.uh_elem()), sh=DArray.from_numpy(P.SH))
    out = alloc_elemental_outputs(m, a, ne)
    stream = torch.cuda.current_stream()

    mixed_out = alloc_elemental_outputs(m, a, ne)

    def step_fp64():
        hdg_elemental(m, a, d_in["dg"], d_in["bf"], d_in["udg"], d_in["uh"], d_in["sh"], out=out,
                      stream=stream, dmaster=dm)

    def step_mixed():
        hdg_elemental(m, a, d_in["dg"], d_in["bf"], d_in["udg"], d_in["uh"], d_in["sh"], out=mixed_out,
                      stream=stream, dmaster=dm, mixed=True)

    for _ in range(args.warmup):
        step_fp64()
        step_mixed()
    torch.cuda.synchronize()
    if int(out.status.numpy().max()) != 0 or int(mixed_out.status.numpy().max()) != 0:
        raise RuntimeError("elemental kernel reported a singular element")
    # accuracy of the mixed form on this step: condensed residual FE vs the FP64 form
    fe_err = float((mixed_out.FE.t - out.FE.t).abs().max() / out.FE.t.abs().max())
    ae_err = float((mixed_out.AE.t - out.AE.t).abs().max() / out.AE.t.abs().max())
    use_mixed = args.precision == "mixed"
    step = step_mixed if use_mixed else step_fp64

    sampler = ClockSampler(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    time.sleep(0.25)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for i in range(args.steps):
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
    t1.record(stream)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    clocks = sampler.stop()
    total_ms = t0.elapsed_time(t1)
    kern_ms = [s.elapsed_time(e) for s, e in ev]
    total_ms = max_over_ranks(total_ms, ws, "cuda")
    ms_per_step = total_ms / args.steps
    value = job_rate(ne, ws, args.steps, total_ms)
    # the other precision, same protocol (no clock sampling)
    other = step_fp64 if use_mixed else step_mixed
    o0, o1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    o0.record(stream)
    for _ in range(args.steps):
        other()
    o1.record(stream)
    torch.cuda.synchronize()
    other_ms = o0.elapsed_time(o1) / args.steps

    line = None
    if rank == 0:
        cnt = element_counts(m.nd, m.npv, m.npf, m.ngv, m.ngf)
        peaks, peak_kind = measured_peaks()
        fp64_peak = measure_fp64_peak(torch)
        avg_kern_s = statistics.mean(kern_ms) * 1e-3
        achieved_tf = cnt["flops"] * ne / avg_kern_s / 1e12
        achieved_gbs = cnt["bytes"] * ne / avg_kern_s / 1e9
        traffic = profile_traffic(f"elemental_kernel_{wl['name']}", "mixed" if use_mixed else "fp64")
        if traffic is not None and (args.n is not None or args.porder is not None):
            traffic = None                           # the summary is for the full-size workload
        roof = {"bound": "tensor", "pipe": "fp64", "achieved": achieved_tf, "peak": fp64_peak,
                "unit": "TFLOP/s", "frac": achieved_tf / fp64_peak,
                "peak_source": "builder-measured: cuBLAS DGEMM 8192^3 timed by bench.py in this run (MEASURED_PEAKS.json, the driver's file, has no FP64 figure)",
                "traffic": traffic, "algorithmic_flops_per_element": cnt["flops"],
                "algorithmic_bytes_per_element": cnt["bytes"],
                "hbm": {"achieved": achieved_gbs, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": achieved_gbs / peaks["hbm_gbs"], "peak_source": peak_kind}}
        out_bytes = sum(x.t.numel() * x.t.element_size() for x in (out.AE, out.FE, out.DUDG, out.DUDG_DUH))
        avail = psutil.virtual_memory().available
        e2e = None
        if out_bytes > 0.5 * avail:
            e2e = {"value": None, "unit": UNIT,
                   "skipped": f"{out_bytes / 1e9:.1f} GB of pinned host outputs > half of the host's free memory"}
        else:
            # end to end through the public host-array entry point (hdgx_elemental_host: pinned host
            # inputs and outputs, the library overlaps uploads, kernel and downloads in chunks),
            # every copy inside the timed region
            from hdg_b200.elemental import alloc_host_outputs, hdg_elemental_host
            h_in = {k: DArray(v.t.cpu().pin_memory(), v.shape) for k, v in d_in.items()}
            h_out = alloc_host_outputs(m, a, ne)

            def e2e_step():
                hdg_elemental_host(m, a, h_in["dg"], h_in["bf"], h_in["udg"], h_in["uh"], h_in["sh"], out=h_out,
                                   stream=stream, dmaster=dm, mixed=use_mixed)
            e2e_step()                                   # warm-up: grows the library's device pool
            ref_out = mixed_out if use_mixed else out
            for k in ("FE", "DUDG", "status"):
                if not torch.equal(getattr(h_out, k).t, getattr(ref_out, k).t.cpu()):
                    raise RuntimeError(f"host-array entry point differs from the device call in {k}")
            e2e_steps = max(2, min(args.steps, 5))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(e2e_steps):
                e2e_step()
            e1.record(stream)
            torch.cuda.synchronize()
            e2e_ms = e0.elapsed_time(e1) / e2e_steps
            # the same copies issued one after another around the device call, for comparison
            # (into the same pinned buffers: C4's outputs alone are 61 GB of host memory)
            h_ser = [h_out.AE.t, h_out.FE.t, h_out.DUDG.t, h_out.DUDG_DUH.t]
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(e2e_steps):
                for k, v in d_in.items():
                    v.t.copy_(h_in[k].t, non_blocking=True)
                step()
                for h, x in zip(h_ser, (out.AE, out.FE, out.DUDG, out.DUDG_DUH)):
                    h.copy_(x.t, non_blocking=True)
            e1.record(stream)
            torch.cuda.synchronize()
            serial_ms = e0.elapsed_time(e1) / e2e_steps
            h2d = sum(v.t.numel() * v.t.element_size() for v in d_in.values())
            d2h = sum(x.t.numel() * x.t.element_size() for x in (h_out.AE, h_out.FE, h_out.DUDG, h_out.DUDG_DUH,
                                                                 h_out.status))
            e2e = {"value": ne / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                   "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                   "call": "hdgx_elemental_host (pinned host arrays, chunked and overlapped)",
                   "d2h_gbs": d2h / (e2e_ms * 1e-3) / 1e9,
                   "serial_copies_ms_per_step": serial_ms}
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            nth = os.cpu_count() or 1
            v, n, dt = cpu_baseline_timed(P, nth, 10.0)
            cpu = {"value": v, "unit": UNIT, "cores": nth, "kind": "port",
                   "sample": f"{n} element evaluations (the workload's elements, repeated) in {dt:.1f} s, C oracle (volint+faceint+schur_uq2 restated from the reference) on {nth} threads",
                   "reference_schur_uq": cpu_reference_schur(P)}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32" if use_mixed else "f64",
            "data": "synthetic (seeded PCG64 state on a generated mesh)",
            "config": {"workload": wl["desc"],
                       "step": f"hdg_elemental over all elements ({'mixed-precision' if use_mixed else 'FP64'} fused kernel)",
                       "elements_per_gpu": ne, "parallelism": f"replicas x{ws} (elements independent)",
                       "l2": f"each step writes {d2h / 1e9:.2f} GB of outputs (> 126 MB L2), evicting the inputs"},
            "roofline": roof, "cpu_baseline": cpu,
            "e2e": e2e,
            "clocks": clocks, "gpu_launches": args.steps,
            "kernel_ms": {"mean": statistics.mean(kern_ms), "min": min(kern_ms), "max": max(kern_ms)},
        }
        fp64_ms = other_ms if use_mixed else ms_per_step
        mixed_ms = ms_per_step if use_mixed else other_ms
        line["precision"] = {
            "value_is": "mixed" if use_mixed else "fp64",
            "fp64": {"value": ne / (fp64_ms * 1e-3), "ms_per_step": fp64_ms},
            "mixed": {"value": ne / (mixed_ms * 1e-3), "ms_per_step": mixed_ms,
                      "FE_rel_err_vs_fp64": fe_err, "AE_rel_err_vs_fp64": ae_err,
                      "scheme": "FP32 local elimination of the Jacobian columns, FP64-refined residual solve, FP64 residuals"},
            "mixed_over_fp64": fp64_ms / mixed_ms,
        }
        # the elemental step's device buffers (C4: two 61 GB output sets) are not needed below
        out = mixed_out = d_in = None
        step = step_fp64 = step_mixed = other = None
        torch.cuda.empty_cache()
        if not args.no_newton and ws == 1:
            line["newton"] = newton_step(P, torch, args)
        if not args.no_buckets and ws == 1:
            line["buckets"] = buckets_mixed_degree(torch, use_mixed)
            if args.config == "c2":
                try:
                    line["tetrahedra"] = tetrahedra_sample(torch)
                except Exception as exc:         # an auxiliary leg: report it, keep the line
                    line["tetrahedra"] = {"error": repr(exc)}
        if not args.no_serve and ws == 1:
            line["serve"] = serve_mix(torch)
            line["serve"]["shared_launch"] = shared_launch(torch)
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def buckets_mixed_degree(torch, mixed, n=181):
    """Mixed-degree workload: 2D Euler M 0.6 + vortex on [0,10]^2, 181x181x2 = 65,522 triangles
    of degree 1-4 (proportions 0.2/0.4/0.3/0.1, seeded), one elemental evaluation of every
    element per step.  The bucketed call (one CUDA graph, degrees concurrent, schedule from
    hdg_b200.autotune) against the plain per-degree launches one after another."""
    from hdg_b200 import configs
    from hdg_b200.autotune import tune_buckets
    from hdg_b200.batch import ElementalBuckets
    from hdg_b200.perfmodel import element_counts
    P = configs.c3(n=n)
    eb = ElementalBuckets(P, mixed=mixed)
    best, grids, results, solo = tune_buckets(eb, reps=3)
    steps = 10
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if best == "per_degree_sequential":
        fn = eb.run_sequential
    else:
        eb.capture()
        fn = eb.replay
    fn()
    torch.cuda.synchronize()
    s.record()
    for _ in range(steps):
        fn()
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / steps
    s.record()
    for _ in range(steps):
        eb.run_sequential()
    e.record()
    torch.cuda.synchronize()
    ms_seq = s.elapsed_time(e) / steps
    if max(eb.statuses()) != 0:
        raise RuntimeError("elemental kernel reported a singular element in the mixed-degree workload")
    flops = sum(element_counts(2, b["master"].npv, b["master"].npf, b["master"].ngv, b["master"].ngf)["flops"] * b["ne"]
                for b in eb.buckets)
    out = {"workload": "2D Euler M=0.6 + vortex, [0,10]^2 181x181x2 = 65522 triangles, p 1-4 (0.2/0.4/0.3/0.1)",
           "elements": eb.ne, "unit": UNIT, "dtype": "f64+f32" if mixed else "f64",
           "per_degree": [{"p": b["p"], "elements": b["ne"], "solo_ms": t} for b, t in zip(eb.buckets, solo)],
           "schedule": best, "grids": grids, "autotune_ms": results,
           "value": eb.ne / (ms * 1e-3), "ms_per_step": ms,
           "per_degree_sequential": {"value": eb.ne / (ms_seq * 1e-3), "ms_per_step": ms_seq},
           "speedup_vs_per_degree": ms_seq / ms, "algorithmic_tflops": flops / (ms * 1e-3) / 1e12,
           "l2": "each step writes the outputs of all 65,522 elements (> 126 MB L2)"}
    del eb
    torch.cuda.empty_cache()
    return out


def tetrahedra_sample(torch, steps=5):
    """The tetrahedral shapes beside the C2 line: one FP64 elemental evaluation of 3D Euler p = 2
    on 16^3 x 6 = 24,576 tets (C4's shape at an eighth of its size) and of 3D Euler and NS p = 3
    on 8^3 x 6 = 3,072 tets; ms and elements/s (CUDA events, 3 warm-up evaluations)."""
    from hdg_b200 import configs
    from hdg_b200.app import make_app
    from hdg_b200.elemental import DArray, DeviceMaster, alloc_elemental_outputs, hdg_elemental
    res = {}
    for tag, n, p, re in (("c4_shape_p2_euler", 16, 2, np.inf), ("p3_euler", 8, 3, np.inf), ("p3_ns_re100", 8, 3, 100.0)):
        P = configs.c4(n=n, porder=p)
        P.app = make_app(3, re=re, minf=0.4, tau=2.0)
        dm = DeviceMaster(P.master)
        dg = DArray.from_numpy(P.mesh.dgnodes)
        bf = DArray.from_numpy(P.mesh.bf, dtype=torch.int32)
        u, uh, sh = DArray.from_numpy(P.UDG), DArray.from_numpy(P.uh_elem()), DArray.from_numpy(P.SH)
        out = alloc_elemental_outputs(P.master, P.app, P.mesh.ne)
        run = lambda: hdg_elemental(P.master, P.app, dg, bf, u, uh, sh, out=out, dmaster=dm)
        for _ in range(3):
            run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            run()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        res[tag] = {"elements": P.mesh.ne, "ms_per_step": ms, "value": P.mesh.ne / (ms * 1e-3), "unit": "elements/s",
                    "status_max": int(out.status.numpy().max())}
        del out
    torch.cuda.empty_cache()
    return res


def serve_mix(torch, count=16, slots=8, ordering="mdf"):
    """Serving: a seeded stream of independent steady solves (2D, n x n x 2 triangles with
    n in 8..20, p in 1..4, Mach 0.3-0.8, half Euler / half NS Re 200-2000, Poisson arrivals at
    20/s) served with continuous admission on per-request streams, against the same requests
    run back to back; solves/s, p50/p99 latency, and whether every result in the mix equals
    its result alone bit for bit."""
    from hdg_b200.serve import Server, request_mix
    kw = dict(nmin=8, nmax=20, pmin=1, pmax=4, rate=20.0)
    seq = request_mix(11, count, **kw)
    s_seq = Server(slots=1, ordering=ordering).serve_sequential(seq)
    conc = request_mix(11, count, **kw)
    s_conc = Server(slots=slots, ordering=ordering).serve(conc)
    same = all(a.UDG is not None and b.UDG is not None and np.array_equal(a.UDG, b.UDG)
               and np.array_equal(a.UH, b.UH) for a, b in zip(seq, conc))
    # capacity: 4x as many requests, all waiting at t = 0 (the arrival rate no longer caps the
    # rate, and no single large request sets the makespan)
    seq2 = request_mix(12, 4 * count, **kw)
    c_seq = Server(slots=1, ordering=ordering).serve_sequential(seq2, realtime=False)
    conc2 = request_mix(12, 4 * count, **kw)
    c_conc = Server(slots=slots, ordering=ordering).serve(conc2, realtime=False)
    # the C5 request distribution (2D, p 1-4, Mach 0.3-0.8, half Euler / half NS Re 200-2000,
    # Poisson 20/s) with the square count truncated to n 24-40 so that both runs fit the bench:
    # 2 x count requests on 2 x slots slots, after one untimed pass of count other requests of the
    # distribution (the library's memory pool grown to the concurrent footprint, every kernel loaded)
    c5kw = dict(nmin=24, nmax=40, pmin=1, pmax=4, rate=20.0)
    c5n, c5slots = 2 * count, 2 * slots
    Server(slots=c5slots, ordering=ordering).serve(request_mix(20, count, **c5kw), realtime=False)
    c5_seq = Server(slots=1, ordering=ordering).serve_sequential(request_mix(21, c5n, **c5kw))
    c5_conc_reqs = request_mix(21, c5n, **c5kw)
    c5_conc = Server(slots=c5slots, ordering=ordering).serve(c5_conc_reqs)
    # the same stream with the running requests' same-degree, same-physics assemblies batched into
    # shared launches (hdgx_solve_combined, 1 ms batching window)
    comb_srv = Server(slots=c5slots, ordering=ordering, combine=True, window_us=1000)
    c5_comb_reqs = request_mix(21, c5n, **c5kw)
    c5_comb = comb_srv.serve(c5_comb_reqs)
    c5_comb["combiner"] = comb_srv.combiner_stats
    c5_comb["identical_to_uncombined"] = all(np.array_equal(a.UDG, b.UDG) and np.array_equal(a.UH, b.UH)
                                             for a, b in zip(c5_conc_reqs, c5_comb_reqs))
    torch.cuda.empty_cache()
    return {"requests": count, "slots": slots, "ordering": ordering, "newton_tol": 1e-10,
            "host_waits": "concurrent runs: blocking-sync events (hdgx_set_host_wait(1)); back to back: CUDA's spinning wait",
            "mix": "2D n x n x 2, n 8-20, p 1-4, M 0.3-0.8, half Euler / half NS Re 200-2000, Poisson 20/s (seed 11)",
            "concurrent": s_conc, "sequential": s_seq, "identical_alone_vs_mix": bool(same),
            "speedup_solves_per_s": s_conc["solves_per_s"] / s_seq["solves_per_s"],
            "capacity": {"note": f"{4 * count} requests of the same distribution (seed 12), all queued at t = 0",
                         "concurrent": c_conc, "sequential": c_seq,
                         "speedup_solves_per_s": c_conc["solves_per_s"] / c_seq["solves_per_s"]},
            "c5_subset": {"mix": f"C5 distribution truncated to n 24-40: {c5n} requests, 2D n x n x 2, p 1-4, "
                                 "M 0.3-0.8, half Euler / half NS Re 200-2000, Poisson 20/s (seed 21)",
                          "slots": c5slots, "warm_up": f"one untimed queued pass of {count} requests (seed 20)",
                          "elements": int(sum(r.problem.mesh.ne for r in c5_conc_reqs)),
                          "concurrent": c5_conc, "sequential": c5_seq, "concurrent_shared_launches": c5_comb,
                          "speedup_solves_per_s": c5_conc["solves_per_s"] / c5_seq["solves_per_s"]}}


def serve_c5(torch, count, slots=16, ordering="mdf"):
    """The C5 serving distribution over its full size range: count requests of 2D n x n x 2
    triangles with n 24-180 (1,152-64,800 elements), p 1-4, Mach 0.3-0.8, half Euler / half NS
    Re 200-2000, Poisson arrivals at 20/s, served with continuous admission on `slots` slots,
    against the same requests back to back.  Newton to 1e-10, MDF BILU(0)-GMRES."""
    from hdg_b200.serve import Server, request_mix
    kw = dict(nmin=24, nmax=180, pmin=1, pmax=4, rate=20.0)
    Server(slots=slots, ordering=ordering).serve(request_mix(40, 8, **dict(kw, nmax=60)), realtime=False)
    from hdg_b200.serve import SolveRequest
    seq_reqs = request_mix(41, count, **kw)
    conc_reqs = [SolveRequest(r.rid, r.problem, arrival=r.arrival) for r in seq_reqs]   # the same inputs
    seq = Server(slots=1, ordering=ordering).serve_sequential(seq_reqs)
    conc = Server(slots=slots, ordering=ordering).serve(conc_reqs)
    same = all(a.UDG is not None and b.UDG is not None and np.array_equal(a.UDG, b.UDG)
               and np.array_equal(a.UH, b.UH) for a, b in zip(seq_reqs, conc_reqs))
    return {"serve_c5": {"mix": f"C5: {count} requests, 2D n x n x 2 with n 24-180, p 1-4, M 0.3-0.8, half Euler / "
                                "half NS Re 200-2000, Poisson 20/s (seed 41)",
                         "elements": int(sum(r.problem.mesh.ne for r in conc_reqs)), "slots": slots,
                         "ordering": ordering, "newton_tol": 1e-10,
                         "concurrent": conc, "sequential": seq, "identical_alone_vs_mix": bool(same),
                         "speedup_solves_per_s": conc["solves_per_s"] / seq["solves_per_s"]}}


def shared_launch(torch, count=24, n=6, p=3, steps=20):
    """Many small independent problems of one degree (24 NS requests on 6 x 6 x 2 triangles at
    p = 3, each with its own Re, Mach and state): one elemental evaluation of all of them per step,
    as ONE segmented launch (hdgx_elemental_shared) against one launch per problem on one stream.
    Outputs are bitwise equal (tests/test_shared_gpu.py)."""
    from hdg_b200.batch import SharedLaunch
    from hdg_b200.serve import request_mix
    rs = request_mix(31, 2 * count, nmin=n, nmax=n, pmin=p, pmax=p)
    sl = SharedLaunch([r.problem for r in rs if r.rid % 2 == 1][:count])
    st = torch.cuda.current_stream()

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    ms_shared = timed(lambda: sl.run(stream=st))
    ms_each = timed(lambda: sl.run_each(stream=st))
    return {"problems": len(sl.items), "elements": sl.ne, "workload": f"{count} NS problems, {n}x{n}x2 triangles, p={p}",
            "shared_ms": ms_shared, "per_problem_ms": ms_each, "speedup": ms_each / ms_shared,
            "shared_elements_per_s": sl.ne / (ms_shared * 1e-3)}


def newton_step(P, torch, args):
    """One full Newton iteration (hdg_solve.m:108-176) on the device, FP64 and mixed:
    elemental + global assembly, BILU(0) factor, GMRES to 1e-10, back-substitution, and the
    line-search re-assembly; elements / (wall time of the iteration, synchronised)."""
    from hdg_b200.elemental import DArray
    from hdg_b200.solve import HDGSolver
    res = {}
    for tag, mixed in (("fp64", False), ("mixed", True)):
        s = HDGSolver(P.master, P.mesh, P.app, mixed=mixed)
        U = DArray.from_numpy(P.UDG); H = DArray.from_numpy(P.UH); S = DArray.from_numpy(P.SH)
        s.solve(U, H, S, tol=1e-10, maxiter=1)            # warm-up (compiles nothing; first-touch)
        U = DArray.from_numpy(P.UDG); H = DArray.from_numpy(P.UH)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rep = s.solve(U, H, S, tol=1e-10, maxiter=1)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        res[tag] = {"value": P.mesh.ne / dt, "unit": UNIT, "s": dt, "gmres_iters": rep.gmres_iters,
                    "gmres_relres": rep.gmres_relres, "residuals": rep.residuals}
        del s
        torch.cuda.empty_cache()
    res["mixed_over_fp64"] = res["mixed"]["value"] / res["fp64"]["value"]
    if not args.no_cpu_baseline:
        res["cpu_baseline"] = cpu_newton_step(P, res["fp64"]["gmres_iters"][0])
    res["note"] = "one Newton iteration incl. initial assembly, BILU(0)-GMRES(20) to 1e-10, back-substitution, line-search re-assembly"
    res["breakdown"] = newton_breakdown(P, torch)
    return res


def newton_breakdown(P, torch):
    """CUDA-event times of the operations of one Newton linear solve (FP64, MDF order)."""
    from hdg_b200.elemental import DArray
    from hdg_b200.solve import HDGSolver
    s = HDGSolver(P.master, P.mesh, P.app)
    U = DArray.from_numpy(P.UDG); H = DArray.from_numpy(P.UH); S = DArray.from_numpy(P.SH)

    def timed(fn, reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    out = {}
    s.assemble(U, H, S)
    out["assemble_ms"] = timed(lambda: s.assemble(U, H, S), 3)
    t0 = time.perf_counter()
    s.ts.bilu0(s.Hg, s.Mg)
    torch.cuda.synchronize()
    out["first_factor_with_mdf_order_ms"] = 1e3 * (time.perf_counter() - t0)
    out["bilu0_factor_ms"] = timed(lambda: s.ts.bilu0(s.Hg, s.Mg), 2)
    x, w = s.ts.empty_vec(), s.ts.empty_vec()
    out["bilu0_apply_ms"] = timed(lambda: s.ts.bilu0_apply(s.Mg, s.Rg, x, w), 10)
    out["matvec_ms"] = timed(lambda: s.ts.matvec(s.Hg, s.Rg, x), 10)
    s.DUH.t.zero_()
    t0 = time.perf_counter()
    gi, _, _, _ = s.ts.gmres(s.Hg, s.Mg, s.Rg, s.DUH, 20, 1e-10, 1000, s.ws)
    torch.cuda.synchronize()
    out["gmres_ms"] = 1e3 * (time.perf_counter() - t0)
    out["gmres_iterations"] = gi
    out["backsub_ms"] = timed(lambda: s.backsub(), 5)
    out["levels"] = int(s.ts.ord.ncolors)
    del s
    torch.cuda.empty_cache()
    return out


if __name__ == "__main__":
    sys.exit(main())
