"""The on-disk state of util/writeBinaryFile.m (single-process branch, lines 14-160): the file
that hands a problem (master tables, app, mesh, UDG, UH and the block-CSR pattern) to the
external C++ solver, and back.

Layout: ``<filename>.bin`` holds float64 values only, each array column-major as MATLAB stores
it, in the order of ``FIELDS``: a 100-entry header ``ndims`` (``HEADER`` maps its 1-based
positions), then the arrays.  Integer arrays (elcon, bf, t2f, perm, cbsr_*) are written as
doubles with the values they hold (1-based where the reference's are).  ``endian`` is
"native", "ieee-le" or "ieee-be" (writeBinaryFile.m's endianType 0, 1, 2).

The reference's util/readBinaryFile.m reads UDG and UH right after the header, which is not
where writeBinaryFile.m puts them; ``read_binary_file`` reads the writer's layout.

App fields the steady HDG app here does not carry take the values of a steady,
single-subdomain problem: morder = porder, torder = nstage = 1, ncq = nc - ncu, ncp = 0,
nch = ncu, ns = 1, no time steps, flags, factors or problem values, zero bcd / bcv, and
permgeom = perm (geometry order = solution order)."""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

# ndims(k) = <expression> of writeBinaryFile.m:17-53
HEADER = {
    1: "mesh.nd", 2: "mesh.ncd", 3: "mesh.nfe", 4: "mesh.nve", 5: "mesh.nvf", 6: "mesh.ne", 7: "mesh.nf",
    8: "mesh.nv", 9: "mesh.ndh", 10: "master.npe", 11: "master.npf", 12: "master.nme", 13: "master.nmf",
    14: "master.nge", 15: "master.ngf", 16: "app.porder", 17: "app.morder", 18: "app.torder",
    19: "app.nstage", 20: "app.nc", 21: "app.ncu", 22: "app.ncq", 23: "app.ncp", 24: "app.nch", 25: "app.ns",
    26: "app.nb", 27: "app.ndt", 28: "app.nparam", 29: "app.nflag", 30: "app.nfactor", 31: "app.nproblem",
    32: "mesh.cbsr_nrows", 33: "mesh.cbsr_nblks", 34: "mesh.maxBlocksPerRow", 35: "mesh.blkSize", 40: "nproc",
}

# the fwrite sequence of writeBinaryFile.m:56-96 (PDG only when app.wave == 1)
FIELDS = [
    "ndims", "master.plocvl", "master.gpvl", "master.gwvl", "master.plocfc", "master.gpfc", "master.gwfc",
    "master.shapvt", "master.shapvg", "master.shapvgdotshapvl", "master.shapft", "master.shapfg",
    "master.shapfgdotshapfc", "master.shapmv", "master.shapmf", "app.bcm(:)", "app.bcs'", "app.bcd(:)",
    "app.bcv'", "app.dt(:)", "app.param(:)", "app.flag(:)", "app.factor(:)", "app.problem(:)",
    "mesh.dgnodes", "mesh.elcon", "mesh.bf", "mesh.t2f", "mesh.perm", "mesh.permgeom", "UDG", "UH", "PDG",
    "mesh.cbsr_rowpts", "mesh.cbsr_colind",
]

_ENDIAN = {"native": "=f8", "ieee-le": "<f8", "ieee-be": ">f8"}


def _shapes(h):
    """Shape of every array in FIELDS from the header values ``h`` (name -> int)."""
    nd, npe, npf, nge, ngf = h["mesh.nd"], h["master.npe"], h["master.npf"], h["master.nge"], h["master.ngf"]
    nme, nmf, ne, nfe, nb = h["master.nme"], h["master.nmf"], h["mesh.ne"], h["mesh.nfe"], h["app.nb"]
    nch = h["app.nch"]
    return {
        "ndims": (100,), "master.plocvl": (npe, nd), "master.gpvl": (nge, nd), "master.gwvl": (nge,),
        "master.plocfc": (npf, nd - 1), "master.gpfc": (ngf, nd - 1), "master.gwfc": (ngf,),
        "master.shapvt": (nge, npe, nd + 1), "master.shapvg": (npe, nge, nd + 1),
        "master.shapvgdotshapvl": (npe * npe, nge, nd + 1), "master.shapft": (ngf, npf, nd),
        "master.shapfg": (npf, ngf, nd), "master.shapfgdotshapfc": (npf * npf, ngf, nd),
        "master.shapmv": (nge, nme, nd + 1), "master.shapmf": (ngf, nmf, nd),
        "app.bcm(:)": (nb,), "app.bcs'": (nch, nb), "app.bcd(:)": (nb,), "app.bcv'": (nch, nb),
        "app.dt(:)": (h["app.ndt"],), "app.param(:)": (h["app.nparam"],), "app.flag(:)": (h["app.nflag"],),
        "app.factor(:)": (h["app.nfactor"],), "app.problem(:)": (h["app.nproblem"],),
        "mesh.dgnodes": (nme, h["mesh.ncd"], ne), "mesh.elcon": (npf * nfe, ne), "mesh.bf": (nfe, ne),
        "mesh.t2f": (ne, nfe), "mesh.perm": (npf, nfe), "mesh.permgeom": (nmf, nfe),
        "UDG": (npe, h["app.nc"], ne), "UH": (nch, h["mesh.ndh"]), "PDG": (npe, h["app.ncu"], ne),
        "mesh.cbsr_rowpts": (h["mesh.cbsr_nrows"] + 1,), "mesh.cbsr_colind": (h["mesh.cbsr_nblks"],),
    }


def _app_list(app, name):
    return np.asarray(getattr(app, name, []), dtype=np.float64).ravel(order="F")


def state_arrays(mesh, master, app, UDG, UH, PDG=None):
    """The header values and the arrays of FIELDS for one problem (name -> ndarray)."""
    nd = master.nd
    npv, npf = master.shapvt.shape[1], master.shapft.shape[1]
    ngv, ngf = master.shapvt.shape[0], master.shapft.shape[0]
    ne, nfe = mesh.t2f.shape
    ncu, nc = app.ncu, app.nc
    rp = np.asarray(mesh.cbsr_rowpts)
    bcm = np.asarray(app.bcm, dtype=np.float64).ravel()
    nb = bcm.size
    bcs = np.asarray(app.bcs, dtype=np.float64).reshape((nb, -1))[:, :ncu] if nb else np.zeros((0, ncu))
    wave = int(getattr(app, "wave", 0))
    h = {
        "mesh.nd": nd, "mesh.ncd": mesh.dgnodes.shape[1], "mesh.nfe": nfe, "mesh.nve": nd + 1, "mesh.nvf": nd,
        "mesh.ne": ne, "mesh.nf": len(rp) - 1, "mesh.nv": np.asarray(mesh.p).shape[0],
        "mesh.ndh": np.asarray(UH).shape[1], "master.npe": npv, "master.npf": npf, "master.nme": npv,
        "master.nmf": npf, "master.nge": ngv, "master.ngf": ngf, "app.porder": master.porder,
        "app.morder": master.porder, "app.torder": int(getattr(app, "torder", 1)),
        "app.nstage": int(getattr(app, "nstage", 1)), "app.nc": nc, "app.ncu": ncu, "app.ncq": nc - ncu,
        "app.ncp": 0, "app.nch": ncu, "app.ns": 1, "app.nb": nb, "app.ndt": _app_list(app, "dt").size,
        "app.nparam": np.asarray(app.param).size, "app.nflag": _app_list(app, "flag").size,
        "app.nfactor": _app_list(app, "factor").size, "app.nproblem": _app_list(app, "problem").size,
        "mesh.cbsr_nrows": len(rp) - 1, "mesh.cbsr_nblks": int(rp[-1]),
        "mesh.maxBlocksPerRow": int(np.diff(rp).max()) if len(rp) > 1 else 0, "mesh.blkSize": ncu * npf,
        "nproc": 1,
    }
    ndims = np.zeros(100)
    for k, name in HEADER.items():
        ndims[k - 1] = h[name]
    perm = np.asarray(master.perm)
    arrays = {
        "ndims": ndims, "master.plocvl": master.plocvl, "master.gpvl": master.gpvl, "master.gwvl": master.gwvl,
        "master.plocfc": master.plocfc, "master.gpfc": master.gpfc, "master.gwfc": master.gwfc,
        "master.shapvt": master.shapvt, "master.shapvg": master.shapvg,
        "master.shapvgdotshapvl": master.shapvgdotshapvl, "master.shapft": master.shapft,
        "master.shapfg": master.shapfg, "master.shapfgdotshapfc": master.shapfgdotshapfc,
        "master.shapmv": master.shapmv, "master.shapmf": master.shapmf,
        "app.bcm(:)": bcm, "app.bcs'": bcs.T, "app.bcd(:)": _app_list(app, "bcd") if hasattr(app, "bcd") else np.zeros(nb),
        "app.bcv'": np.asarray(getattr(app, "bcv", np.zeros((nb, ncu)))).reshape((nb, -1)).T,
        "app.dt(:)": _app_list(app, "dt"), "app.param(:)": np.asarray(app.param, dtype=np.float64).ravel(order="F"),
        "app.flag(:)": _app_list(app, "flag"), "app.factor(:)": _app_list(app, "factor"),
        "app.problem(:)": _app_list(app, "problem"),
        "mesh.dgnodes": mesh.dgnodes, "mesh.elcon": mesh.elcon, "mesh.bf": mesh.bf, "mesh.t2f": mesh.t2f,
        "mesh.perm": perm, "mesh.permgeom": perm, "UDG": UDG, "UH": UH,
        "mesh.cbsr_rowpts": rp, "mesh.cbsr_colind": mesh.cbsr_colind,
    }
    if wave:
        if PDG is None:
            raise ValueError("app.wave == 1 needs PDG")
        arrays["PDG"] = PDG
    shapes = _shapes(h)
    for name, a in arrays.items():
        a = np.asarray(a, dtype=np.float64)
        if a.size != int(np.prod(shapes[name])):
            raise ValueError(f"{name}: {a.size} values, the header implies {shapes[name]}")
        arrays[name] = a.reshape(shapes[name], order="F")
    return h, arrays


def write_binary_file(filename, mesh, master, app, UDG, UH, PDG=None, endian="native"):
    """util/writeBinaryFile.m with nproc = 1: writes ``<filename>.bin``; returns its path."""
    h, arrays = state_arrays(mesh, master, app, UDG, UH, PDG)
    dt = np.dtype(_ENDIAN[endian])
    path = Path(str(filename) + ".bin")
    with open(path, "wb") as f:
        for name in FIELDS:
            if name in arrays:
                f.write(np.asarray(arrays[name], dtype=dt).ravel(order="F").tobytes())
    return path


@dataclass
class BinaryState:
    header: dict = field(default_factory=dict)     # HEADER name -> int
    arrays: dict = field(default_factory=dict)     # FIELDS name -> ndarray (MATLAB shapes)


def read_binary_file(filename, endian="native", wave=False):
    """Read the layout ``write_binary_file`` / writeBinaryFile.m (nproc = 1) writes.  ``wave``
    says whether the file holds PDG (app.wave == 1; the header does not record it)."""
    dt = np.dtype(_ENDIAN[endian])
    raw = np.fromfile(str(filename) + ".bin", dtype=dt).astype(np.float64)
    if raw.size < 100:
        raise ValueError("not a writeBinaryFile state: shorter than its 100-value header")
    h = {name: int(round(raw[k - 1])) for k, name in HEADER.items()}
    shapes = _shapes(h)
    out, pos = {}, 0
    for name in FIELDS:
        if name == "PDG" and not wave:
            continue
        n = int(np.prod(shapes[name]))
        if pos + n > raw.size:
            raise ValueError(f"file ends inside {name}")
        out[name] = raw[pos:pos + n].reshape(shapes[name], order="F")
        pos += n
    if pos != raw.size:
        raise ValueError(f"{raw.size - pos} values after the last field")
    return BinaryState(h, out)
