"""ctypes binding of libhdgx.so (the C ABI declared in include/hdgx.h).

The library is required: importing the compute entry points without it, or calling them
without a CUDA device, raises.  There is no CPU fallback in this package.
"""
from __future__ import annotations

import ctypes as ct
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libhdgx.so"
HDGX_MAX_BND = 16

_dp = ct.c_void_p


class HdgxMaster(ct.Structure):
    _fields_ = [("nd", ct.c_int), ("porder", ct.c_int), ("npv", ct.c_int), ("npf", ct.c_int),
                ("nfe", ct.c_int), ("ngv", ct.c_int), ("ngf", ct.c_int),
                ("shapvt", _dp), ("shapvg", _dp), ("shapmv", _dp), ("shapft", _dp),
                ("shapfg", _dp), ("shapmf", _dp), ("perm", _dp)]


class HdgxApp(ct.Structure):
    _fields_ = [("nd", ct.c_int), ("ncu", ct.c_int), ("nc", ct.c_int), ("localsolve", ct.c_int),
                ("getdqdg", ct.c_int), ("fc_q", ct.c_double), ("fc_u", ct.c_double), ("tdep", ct.c_int),
                ("param", ct.c_double * 8), ("nbnd", ct.c_int), ("bcm", ct.c_int * HDGX_MAX_BND),
                ("bcs", ct.c_double * (HDGX_MAX_BND * 5)), ("fbou", ct.c_int)]


class HdgxBsr(ct.Structure):
    _fields_ = [("nf", ct.c_int), ("bs", ct.c_int), ("nnzb", ct.c_longlong), ("rowpts", _dp), ("colind", _dp),
                ("ncolors", ct.c_int), ("color_ptr", _dp), ("color_rows", _dp), ("pos", _dp), ("sched", _dp),
                ("sweep_plan", _dp), ("sweep_maxd", ct.c_int)]


class HdgxElemBucket(ct.Structure):
    _fields_ = [("master", _dp), ("app", _dp), ("ne", ct.c_int), ("dgnodes", _dp), ("bf", _dp), ("UDG", _dp),
                ("UH", _dp), ("SH", _dp), ("AE", _dp), ("FE", _dp), ("DUDG", _dp), ("DUDG_DUH", _dp),
                ("status", _dp), ("grid", ct.c_int)]


HDGX_SOLVE_MAXIT = 16


class HdgxMesh(ct.Structure):
    _fields_ = [("ne", ct.c_int), ("nf", ct.c_int), ("dgnodes", _dp), ("bf", _dp), ("elcon", _dp), ("t2f", _dp),
                ("rowpts", _dp), ("colind", _dp)]


class HdgxSolveOpts(ct.Structure):
    _fields_ = [("ordering", ct.c_int), ("mixed", ct.c_int), ("restart", ct.c_int), ("maxiter", ct.c_int),
                ("tol", ct.c_double), ("gmres_tol", ct.c_double), ("gmres_maxit", ct.c_int)]


class HdgxSolveReport(ct.Structure):
    _fields_ = [("iterations", ct.c_int), ("converged", ct.c_int), ("ncolors", ct.c_int),
                ("residuals", ct.c_double * (HDGX_SOLVE_MAXIT + 1)), ("alphas", ct.c_double * HDGX_SOLVE_MAXIT),
                ("gmres_iters", ct.c_int * HDGX_SOLVE_MAXIT), ("gmres_relres", ct.c_double * HDGX_SOLVE_MAXIT),
                ("graph_assemblies", ct.c_int)]


class HdgxAssemblyMap(ct.Structure):
    _fields_ = [("blk_e", _dp), ("blk_ab", _dp), ("blk_row", _dp), ("face_e", _dp), ("face_a", _dp)]


_LIB = None


class HdgxError(RuntimeError):
    pass


def lib():
    """Load libhdgx.so (building it first when the sources are newer)."""
    global _LIB
    if _LIB is None:
        from . import build as _build
        if _build.needs_build():
            _build.build()
        if not LIB_PATH.exists():
            raise HdgxError(f"{LIB_PATH} is missing; run python -m hdg_b200.build")
        L = ct.CDLL(str(LIB_PATH))
        _declare(L)
        _LIB = L
    return _LIB


def _declare(L):
    i, d, v, p = ct.c_int, ct.c_double, ct.c_void_p, ct.POINTER
    L.hdgx_version.restype = i
    L.hdgx_set_host_wait.restype = i
    L.hdgx_set_host_wait.argtypes = [i]
    L.hdgx_get_host_wait.restype = i
    L.hdgx_get_host_wait.argtypes = []
    L.hdgx_status_str.restype = ct.c_char_p
    L.hdgx_status_str.argtypes = [i]
    L.hdgx_status_count.restype = i
    L.hdgx_status_count.argtypes = [v, i, v]
    L.hdgx_elemental.restype = i
    L.hdgx_elemental.argtypes = [p(HdgxMaster), p(HdgxApp), i] + [v] * 10 + [v]
    L.hdgx_elemental_mixed.restype = i
    L.hdgx_elemental_mixed.argtypes = [p(HdgxMaster), p(HdgxApp), i] + [v] * 10 + [v]
    L.hdgx_elemental_host.restype = i
    L.hdgx_elemental_host.argtypes = [p(HdgxMaster), p(HdgxApp), i] + [v] * 10 + [i, i, v]
    L.hdgx_schur_uq.restype = i
    L.hdgx_schur_uq.argtypes = [i] * 5 + [v] * 15 + [v]
    L.hdgx_getq.restype = i
    L.hdgx_getq.argtypes = [p(HdgxMaster), p(HdgxApp), i] + [v] * 7 + [v]
    L.hdgx_residual.restype = i
    L.hdgx_residual.argtypes = [p(HdgxMaster), p(HdgxApp), i] + [v] * 7 + [v]
    L.hdgx_schur_uq_adjoint.restype = i
    L.hdgx_schur_uq_adjoint.argtypes = [i] * 5 + [v] * 15 + [v]
    L.hdgx_schur_u_adjoint.restype = i
    L.hdgx_schur_u_adjoint.argtypes = [i] * 5 + [v] * 11 + [v]
    L.hdgx_schur_u.restype = i
    L.hdgx_schur_u.argtypes = [i] * 5 + [v] * 11 + [v]
    B, M = p(HdgxBsr), p(HdgxAssemblyMap)
    L.hdgx_gather_uh.restype = i
    L.hdgx_gather_uh.argtypes = [i, i, i, v, v, v, v]
    L.hdgx_globalassembly.restype = i
    L.hdgx_globalassembly.argtypes = [B, M, i, i, i, v, v, v, v, v, v]
    L.hdgx_block_norms.restype = i
    L.hdgx_block_norms.argtypes = [B, v, v, v]
    L.hdgx_mdf_ordering.restype = i
    L.hdgx_mdf_ordering.argtypes = [i, v, v, v, v, v]
    L.hdgx_level_schedule.restype = i
    L.hdgx_level_schedule.argtypes = [i, v, v, v, v, v, v]
    L.hdgx_sweep_plan.restype = i
    L.hdgx_sweep_plan.argtypes = [i, v, v, i, v, v, v, v, p(i)]
    L.hdgx_matvec.restype = i
    L.hdgx_matvec.argtypes = [B, v, v, v, v]
    L.hdgx_bilu0_factor.restype = i
    L.hdgx_bilu0_factor.argtypes = [B, v, v, v]
    L.hdgx_bilu0_apply.restype = i
    L.hdgx_bilu0_apply.argtypes = [B, v, v, v, v, v]
    L.hdgx_gmres_workspace_bytes.restype = ct.c_size_t
    L.hdgx_gmres_workspace_bytes.argtypes = [B, i]
    L.hdgx_gmres_bilu0.restype = i
    L.hdgx_gmres_bilu0.argtypes = [B, v, v, v, v, i, d, i, p(i), p(i), p(d), v, v, v]
    L.hdgx_bilu0_to_f32.restype = i
    L.hdgx_bilu0_to_f32.argtypes = [B, v, v, v]
    L.hdgx_gmres_bilu0_mixed.restype = i
    L.hdgx_gmres_bilu0_mixed.argtypes = [B, v, v, v, v, i, d, i, p(i), p(i), p(d), v, v, v]
    L.hdgx_gmres_bilu0_noalloc.restype = i
    L.hdgx_gmres_bilu0_noalloc.argtypes = [B, v, v, v, v, i, d, i, p(i), p(i), p(d), v, v]
    L.hdgx_backsub.restype = i
    L.hdgx_backsub.argtypes = [i, i, i, i, i, v, v, v, v, v, v]
    L.hdgx_solve.restype = i
    L.hdgx_solve.argtypes = [p(HdgxMaster), p(HdgxApp), p(HdgxMesh), v, v, v, p(HdgxSolveOpts), p(HdgxSolveReport), v]
    L.hdgx_elemental_buckets.restype = i
    L.hdgx_elemental_buckets.argtypes = [i, v, i, v]
    L.hdgx_elemental_shared.restype = i
    L.hdgx_elemental_shared.argtypes = [i, v, i, v]
    L.hdgx_elemental_shared_max.restype = i
    L.hdgx_elemental_shared_max.argtypes = []
    L.hdgx_combiner_create.restype = i
    L.hdgx_combiner_create.argtypes = [i, p(v)]
    L.hdgx_combiner_destroy.restype = i
    L.hdgx_combiner_destroy.argtypes = [v]
    L.hdgx_combiner_stats.restype = i
    L.hdgx_combiner_stats.argtypes = [v, p(ct.c_longlong), p(ct.c_longlong), p(ct.c_longlong)]
    L.hdgx_combiner_times.restype = i
    L.hdgx_combiner_times.argtypes = [v, p(d), p(d)]
    L.hdgx_solve_combined.restype = i
    L.hdgx_solve_combined.argtypes = [p(HdgxMaster), p(HdgxApp), p(HdgxMesh), v, v, v, p(HdgxSolveOpts),
                                      p(HdgxSolveReport), v, v]
    L.hdgx_arraymul.restype = i
    L.hdgx_arraymul.argtypes = [i, i, i, i, i, i, v, v, v, v]
    L.hdgx_dense_block_system.restype = i
    L.hdgx_dense_block_system.argtypes = [B, v, v, i, v, v, v, v, v]
    L.hdgx_dense_matvec.restype = i
    L.hdgx_dense_matvec.argtypes = [i, i, i, v, v, v, v, v]
    L.hdgx_gmres_dense_workspace_bytes.restype = ct.c_size_t
    L.hdgx_gmres_dense_workspace_bytes.argtypes = [i, i, i]
    L.hdgx_gmres_dense.restype = i
    L.hdgx_gmres_dense.argtypes = [i, i, i, v, v, v, v, i, d, i, p(i), p(i), p(d), v, v, v]
    _declare_optional(L)


_OPTIONAL = {}


def _declare_optional(L):
    """Entry points added after the elemental kernel; declared when present."""
    i, v = ct.c_int, ct.c_void_p
    for name, res, args in _OPTIONAL.values():
        if hasattr(L, name):
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args


def check(rc, what):
    if rc != 0:
        msg = lib().hdgx_status_str(rc).decode()
        raise HdgxError(f"{what} failed with status {rc}: {msg}")
