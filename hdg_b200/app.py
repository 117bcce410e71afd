"""Application (physics) description and the seeded synthetic initial states.

``App`` mirrors the fields of the reference's ``app`` struct that the elemental path reads
(``kernel/volint.m:12-23``, ``kernel/faceint.m:14-26``, defaults ``kernel/hdg_solve.m:37-60``):
``nd, ncu, nc, arg(param), bcm, bcs, localsolve, fc_q, fc_u, tdep, getdqdg``.

Physics is the compressible Navier--Stokes family of ``application/FM/ns`` with
``param = [gam, epslm, Re, Pr, Minf, tau]`` (``problem/ns/ns_naca.m:36``).  Euler runs
through the same (u,q) form with ``Re = inf`` (every viscous and heat-flux term carries a
factor ``1/Re``, ``application/FM/ns/flux2d.m:30``), so the local block is ``npv*nc``.

Boundary types (``bcm``) are the case labels of the ``fbou.m`` of the app's physics folder
(``fbou``): ``"ns"`` (``application/FM/ns/fbou.m``, ``fbou3d.m``) has 1 far field (Roe matrices
of ``getan.m``), 2 adiabatic wall, 3 isothermal wall, 4 prescribed pressure, 5 periodic
(= fhat), 6 Dirichlet ``fh = uh - uinf`` (``fbou.m:111-114``); ``"euler"``
(``application/FM/euler/fbou.m``) has 1 far field (local Lax-Friedrichs), 2 slip wall, 3 and 4
prescribed pressure, 5 density and energy extrapolated, and 6 Dirichlet as ``"ns"``.  Euler
apps (``Re = inf``) take the ``"euler"`` family, as the reference's Euler drivers do
(``problem/euler/euler_trefftz.m:3`` puts ``application/FM/euler`` on the path).

The synthetic states stand in for the reference's driver scripts (``problem/euler/
euler_trefftz.m:14-19`` freestream; seeded perturbations with a PCG64 generator).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

BC_FARFIELD = 1
BC_WALL = 2
BC_PERIODIC = 5
BC_DIRICHLET = 6


@dataclass
class App:
    nd: int
    param: np.ndarray                 # [gam, epslm, Re, Pr, Minf, tau]
    bcm: np.ndarray                   # [nbnd] boundary type per boundary index
    bcs: np.ndarray                   # [nbnd, ncu] boundary state per boundary index
    localsolve: int = 1
    fc_q: float = 1.0
    fc_u: float = 0.0
    tdep: int = 0
    getdqdg: int = 1
    name: str = "ns"
    denseblock: int = 0               # hdg_solve.m:43-45: 1 = dense face-block GMRES (gmres.m)
    fbou: str = "ns"                  # fbou.m family: "ns" (application/FM/ns) or "euler" (application/FM/euler)

    @property
    def ncu(self):
        return self.nd + 2

    @property
    def nc(self):
        return self.ncu * (self.nd + 1) if self.localsolve else self.ncu

    @property
    def nch(self):
        return self.ncu

    @property
    def inviscid(self):
        return not np.isfinite(self.param[2])


def freestream(nd, gam, minf, alpha=0.0):
    """Conserved freestream state with rho = 1, |u| = 1, p = 1/(gam Minf^2)."""
    pinf = 1.0 / (gam * minf * minf)
    if nd == 2:
        u = np.array([np.cos(alpha), np.sin(alpha)])
    else:
        u = np.array([np.cos(alpha), np.sin(alpha), 0.0])
    return np.concatenate([[1.0], u, [pinf / (gam - 1.0) + 0.5]])


def make_app(nd, gam=1.4, re=np.inf, pr=0.72, minf=0.5, tau=2.0, nbnd=None, alpha=0.0):
    nbnd = nbnd if nbnd is not None else (4 if nd == 2 else 6)
    ui = freestream(nd, gam, minf, alpha)
    return App(nd=nd, param=np.array([gam, 0.0, re, pr, minf, tau], dtype=np.float64),
               bcm=np.full(nbnd, BC_DIRICHLET, dtype=np.int64),
               bcs=np.tile(ui, (nbnd, 1)), name="euler" if not np.isfinite(re) else "ns",
               fbou="euler" if not np.isfinite(re) else "ns")


def _prim_to_cons(rho, vel, p, gam):
    e = p / (gam - 1.0) + 0.5 * rho * np.sum(vel * vel, axis=0)
    return np.concatenate([rho[None], rho[None] * vel, e[None]], axis=0)


def state_vortex(dgnodes, gam, minf, seed, strength=5.0, lo=3.0, hi=7.0):
    """Freestream + isentropic vortex of ``strength`` centred uniformly in ``[lo,hi]^2``."""
    rng = np.random.Generator(np.random.PCG64(seed))
    xc, yc = rng.uniform(lo, hi, size=2)
    x, y = dgnodes[:, 0, :], dgnodes[:, 1, :]
    r2 = (x - xc) ** 2 + (y - yc) ** 2
    f = np.exp(0.5 * (1.0 - r2))
    b = strength / (2.0 * np.pi)
    u = 1.0 - b * (y - yc) * f
    v = b * (x - xc) * f
    tinf = 1.0 / (gam * minf * minf)
    temp = tinf - (gam - 1.0) * strength ** 2 / (8.0 * gam * np.pi ** 2) * np.exp(1.0 - r2)
    rho = (temp / tinf) ** (1.0 / (gam - 1.0))
    p = rho * temp
    return _prim_to_cons(rho, np.stack([u, v]), p, gam)      # [ncu, npv, ne]


def state_fourier(dgnodes, nd, gam, minf, seed, nmodes, amp, field_="velocity"):
    """Freestream + a seeded sum of smooth Fourier modes (std ``amp`` of the freestream)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    x = [dgnodes[:, d, :] for d in range(nd)]
    span = [max(1e-12, float(xd.max() - xd.min())) for xd in x]
    k = rng.integers(1, 4, size=(nmodes, nd))
    ph = rng.uniform(0.0, 2.0 * np.pi, size=(nmodes, nd + 1))
    a = rng.normal(size=(nmodes, nd + 1))
    pert = np.zeros((nd + 1,) + x[0].shape)
    for m in range(nmodes):
        arg = sum(2.0 * np.pi * k[m, d] * x[d] / span[d] for d in range(nd))
        for c in range(nd + 1):
            pert[c] += a[m, c] * np.sin(arg + ph[m, c])
    pert *= amp / max(1e-300, np.sqrt(np.mean(pert ** 2)))
    rho = np.ones_like(x[0])
    vel = np.zeros((nd,) + x[0].shape)
    vel[0] = 1.0
    p = np.full_like(x[0], 1.0 / (gam * minf * minf))
    if field_ == "velocity":
        vel = vel + pert[:nd]
    else:
        rho = rho * (1.0 + pert[0])
    return _prim_to_cons(rho, vel, p, gam)


def init_udg(ucons, nc):
    """UDG[npv, nc, ne] with u = ``ucons`` and q = 0."""
    ncu, npv, ne = ucons.shape
    udg = np.zeros((npv, nc, ne))
    udg[:, :ncu, :] = np.transpose(ucons, (1, 0, 2))
    return udg


def inituhat(perm, elcon, udg, ncu, nsiz):
    """util/inituhat.m:1-28: trace initialised to the average of the element traces."""
    npf, nfe = perm.shape
    ne = udg.shape[2]
    idx = perm.reshape(-1, order="F") - 1                      # [npf*nfe]
    vals = udg[idx, :ncu, :]                                   # [npf*nfe, ncu, ne]
    uh = np.zeros((ncu, nsiz))
    cnt = np.zeros(nsiz)
    ec = elcon - 1                                             # [npf*nfe, ne]
    for a in range(ncu):
        np.add.at(uh[a], ec.ravel(order="F"), vals[:, a, :].ravel(order="F"))
    np.add.at(cnt, ec.ravel(order="F"), 1.0)
    return uh / cnt[None, :]


def gather_uh(uh, elcon):
    """Element-gathered trace ``UH[ncu, ndf, ne] = UH(:, elcon)`` (hdg_assemble.m:34)."""
    ncu = uh.shape[0]
    ndf, ne = elcon.shape
    return uh[:, elcon - 1].reshape(ncu, ndf, ne)
