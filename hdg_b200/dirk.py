"""Diagonally implicit Runge-Kutta time stepping (kernel/hdg_solve_dirk.m) on the GPU solve.

Each stage is one steady HDG solve (``hdg_solve``: fused elemental kernel, BILU(0)-GMRES,
Newton) of the time-dependent residual of volint.m:180-221: the elemental kernel adds the
source ``SH_u - fc_u u`` and its Jacobian ``-fc_u`` on the u components (``app.tdep = 1``),
with ``fc_u = d(s, s)`` and the stage source ``SH`` built from the step's start state and the
earlier stages' solutions as hdg_solve_dirk.m builds SDG.

As the reference does, every stage first forms its source SDG from the current UDG and then
resets the q components of UDG with getq.m (``hdgx_getq`` on the GPU); the reference writes
them as ``UDG(:,4:9,:)``, i.e. for a 3-component model, here they are the components
``ncu+1:nc``.  ``app.wave`` (fc_q = fc_u and the PDG auxiliary variable) is not supported.
"""
from __future__ import annotations

import copy
import math

import numpy as np

from .app import gather_uh
from .elemental import getq
from .solve import hdg_solve


def dirk_coefficients(nstage, torder):
    """dirkcoeff of kernel/hdg_solve_dirk.m: the Butcher tableau (a, b, t) of the
    (stages, order) scheme, returned as d = inv(a), c = b inv(a) and t."""
    if (nstage, torder) == (1, 1):
        a, b, t = [[1.0]], [1.0], [1.0]
    elif (nstage, torder) == (1, 2):
        a, b, t = [[0.5]], [1.0], [0.5]
    elif (nstage, torder) == (2, 2):
        g = 1.0 - 0.5 * math.sqrt(2.0)
        a, b, t = [[g, 0.0], [0.5 * math.sqrt(2.0), g]], [0.5 * math.sqrt(2.0), g], [g, 1.0]
    elif (nstage, torder) == (2, 3):
        g = 0.5 + 0.5 / math.sqrt(3.0)
        a, b, t = [[g, 0.0], [-1.0 / math.sqrt(3.0), g]], [0.5, 0.5], [g, 0.5 - 0.5 / math.sqrt(3.0)]
    elif (nstage, torder) == (3, 3):
        a1 = 0.4358665215
        t1 = (1.0 + a1) / 2.0
        b1 = -(6.0 * a1 ** 2 - 16.0 * a1 + 1.0) / 4.0
        b2 = (6.0 * a1 ** 2 - 20.0 * a1 + 5.0) / 4.0
        a, b, t = [[a1, 0.0, 0.0], [t1 - a1, a1, 0.0], [b1, b2, a1]], [b1, b2, a1], [a1, t1, 1.0]
    elif (nstage, torder) == (3, 4):
        a1 = 2.0 * math.cos(math.pi / 18.0) / math.sqrt(3.0)
        h = 0.5 * (1.0 + a1)
        a = [[h, 0.0, 0.0], [-0.5 * a1, h, 0.0], [1.0 + a1, -(1.0 + 2.0 * a1), h]]
        b = [1.0 / (6.0 * a1 ** 2), 1.0 - 1.0 / (3.0 * a1 ** 2), 1.0 / (6.0 * a1 ** 2)]
        t = [h, 0.5, 0.5 * (1.0 - a1)]
    else:
        raise ValueError(f"no DIRK scheme with {nstage} stages of order {torder} "
                         "(schemes: (1,1) (1,2) (2,2) (2,3) (3,3) (3,4))")
    a = np.array(a, dtype=np.float64)
    d = np.linalg.inv(a)
    return d, np.array(b, dtype=np.float64) @ d, np.array(t, dtype=np.float64)


def stage_source(d, s, UDG, stage_solutions, prev_source):
    """SDG of hdg_solve_dirk.m for stage s (0-based) from the step's start state UDG, the
    earlier stages' solutions and the previous stage's source."""
    if s == 0:
        return d[0, 0] * UDG
    if s == 1:
        return (d[1, 0] + d[1, 1]) * UDG - d[1, 0] * stage_solutions[0]
    if s == 2:
        return ((d[2, 0] + d[2, 1] + d[2, 2]) * UDG
                - (d[2, 0] / d[1, 0]) * ((d[1, 0] + d[1, 1]) * UDG - prev_source)
                - d[2, 1] * stage_solutions[1])
    raise ValueError("hdg_solve_dirk.m defines the stage sources of at most 3 stages")


def hdg_solve_dirk(master, mesh, app, UDG, UH, time, dt, nstage, torder, tol=1e-10, maxiter=16,
                   gmres_tol=1e-10, restart=20, ordering=None, mixed=False):
    """One time step of kernel/hdg_solve_dirk.m from (UDG, UH) at ``time`` to ``time + dt``:
    returns (Un, Hn, reports) as host arrays, reports holding each stage's Newton report."""
    if getattr(app, "wave", 0):
        raise ValueError("app.wave (the PDG auxiliary variable) is not supported")
    d, c, t = dirk_coefficients(nstage, torder)
    d = d / dt
    UDG = np.asarray(UDG, dtype=np.float64)
    UH = np.asarray(UH, dtype=np.float64)
    Un = (1.0 - c.sum()) * UDG
    Hn = (1.0 - c.sum()) * UH
    sols, reports, SDG = [], [], None
    ncu = app.ncu
    UHe = gather_uh(UH, mesh.elcon)
    for s in range(nstage):
        SDG = stage_source(d, s, UDG, sols, SDG)
        sapp = copy.copy(app)
        sapp.fc_u, sapp.fc_q, sapp.tdep = float(d[s, s]), 1.0, 1
        sapp.time = time + dt * t[s]
        Q, _ = getq(master, sapp, mesh.dgnodes, mesh.bf, UDG, UHe, None, sapp.fc_q)
        UDG = np.array(UDG, copy=True)
        UDG[:, ncu:, :] = Q.numpy()
        Us, Hs, rep = hdg_solve(master, mesh, sapp, UDG, UH, SDG, tol=tol, maxiter=maxiter, gmres_tol=gmres_tol,
                                restart=restart, ordering=ordering, mixed=mixed)
        sols.append(Us)
        reports.append(rep)
        Un = Un + c[s] * Us
        Hn = Hn + c[s] * Hs
    return Un, Hn, reports
