"""The synthetic workloads (seeded; no public dataset is involved).

* ``c1``: 2D steady Euler, [0,10]^2, 16x16 squares x 2 triangles = 512 elements, p = 2,
  Mach 0.5 freestream + isentropic vortex of strength 5 centred uniformly in [3,7]^2,
  Dirichlet freestream on all four sides.
* ``c2``: 2D steady Navier--Stokes, Re 1000, Pr 0.72, Mach 0.3, [0,1]^2, 128x128 squares x
  2 = 32,768 elements, p = 3, freestream + Gaussian velocity perturbation (std 1 %, 8 smooth
  Fourier modes).
* ``c4``: 3D steady Euler on tetrahedra, unit cube, 32^3 cubes x 6 = 196,608 elements,
  p = 2, Mach 0.4 + 1 % density perturbation of 6 Fourier modes.
* ``c3``: 2D steady Euler, [0,10]^2, 181x181 squares x 2 = 65,522 elements, each of degree
  p in {1, 2, 3, 4} drawn from the seed with proportions 0.2 / 0.4 / 0.3 / 0.1, Mach 0.6
  freestream + vortex.  The reference defines no mixed-degree coupling, so every degree is a
  bucket of elements evaluated as on the uniform-degree mesh of the same triangulation
  (``MixedDegreeProblem``); the element work is what is measured.
``n`` overrides the number of squares / cubes per side (smaller parity cases).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .app import App, gather_uh, init_udg, inituhat, make_app, state_fourier, state_vortex
from .master import Master, mkmaster
from .mesh import Mesh, mkmesh_cube, mkmesh_square


@dataclass
class Problem:
    name: str
    master: Master
    mesh: Mesh
    app: App
    UDG: np.ndarray      # [npv, nc, ne]
    UH: np.ndarray       # [ncu, nsiz]
    SH: np.ndarray       # [npv, nc, ne]

    def uh_elem(self, UH=None):
        return gather_uh(self.UH if UH is None else UH, self.mesh.elcon)


def _finish(name, master, mesh, app, ucons):
    udg = init_udg(ucons, app.nc)
    uh = inituhat(master.perm, mesh.elcon, udg, app.ncu, mesh.nsiz)
    sh = np.zeros_like(udg)
    return Problem(name, master, mesh, app, udg, uh, sh)


def c1(seed=0, n=16, porder=2):
    mesh = mkmesh_square(n + 1, n + 1, porder, 0, 10.0, 10.0)
    master = mkmaster(2, porder, 2 * porder)
    app = make_app(2, re=np.inf, minf=0.5, tau=2.0)
    u = state_vortex(mesh.dgnodes, 1.4, 0.5, seed)
    return _finish("c1", master, mesh, app, u)


def c2(seed=0, n=128, porder=3):
    mesh = mkmesh_square(n + 1, n + 1, porder, 0, 1.0, 1.0)
    master = mkmaster(2, porder, 2 * porder)
    app = make_app(2, re=1000.0, pr=0.72, minf=0.3, tau=2.0)
    u = state_fourier(mesh.dgnodes, 2, 1.4, 0.3, seed, 8, 0.01, "velocity")
    return _finish("c2", master, mesh, app, u)


def c4(seed=0, n=32, porder=2):
    mesh = mkmesh_cube(n + 1, n + 1, n + 1, porder)
    master = mkmaster(3, porder, 2 * porder)
    app = make_app(3, re=np.inf, minf=0.4, tau=2.0)
    u = state_fourier(mesh.dgnodes, 3, 1.4, 0.4, seed, 6, 0.01, "density")
    return _finish("c4", master, mesh, app, u)


@dataclass
class MixedDegreeProblem:
    name: str
    degree: np.ndarray            # [ne] degree of every element
    buckets: list                 # [(p, Problem on the uniform-degree mesh, element indices)]

    @property
    def ne(self):
        return int(self.degree.shape[0])


def c3(seed=0, n=181, degrees=(1, 2, 3, 4), proportions=(0.2, 0.4, 0.3, 0.1)):
    rng = np.random.Generator(np.random.PCG64(seed))
    ne = 2 * n * n
    deg = rng.choice(np.asarray(degrees), size=ne, p=np.asarray(proportions))
    buckets = []
    for p in degrees:
        idx = np.nonzero(deg == p)[0]
        if idx.size == 0:
            continue
        mesh = mkmesh_square(n + 1, n + 1, p, 0, 10.0, 10.0)
        master = mkmaster(2, p, 2 * p)
        app = make_app(2, re=np.inf, minf=0.6, tau=2.0)
        u = state_vortex(mesh.dgnodes, 1.4, 0.6, seed)
        buckets.append((p, _finish(f"c3-p{p}", master, mesh, app, u), idx))
    return MixedDegreeProblem("c3", deg, buckets)


def by_name(name, **kw):
    return {"c1": c1, "c2": c2, "c3": c3, "c4": c4}[name](**kw)
