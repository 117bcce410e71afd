"""Generate the committed golden fixtures from the reference (run in a tree that has it).

* master_tri_p2.npz  -- master/testpython.mat (p=2, pgauss=4, triangle), fields as stored.
* master_seg_p4.npz  -- the face (segment) tables of the p=4 quadrilateral master stored in
                        problem/burgers/results.mat: plocfc, gpfc, gwfc, shapfc.
* ref_physics.npz    -- outputs of the reference's generated point kernels
                        application/FM/ns/{flux,fhat}_ns{2,3}d.c and application/FM/euler/
                        {flux,fhat}_euler{2,3}d.c (compiled into oracle/_ref)
                        on seeded random states.
* ref_schur.npz      -- outputs of the reference MEX sources kernel/schur_uq.c and
                        kernel/schur_u.c (compiled into oracle/_ref with the MEX emulation)
                        on the elemental blocks of a 2D Euler p=2 case (8 elements) and a
                        2D Navier-Stokes p=3 case (8 elements).
* ref_schur_adjoint.npz -- outputs of kernel/schur_uq_adjoint.c and kernel/schur_u_adjoint.c
                        (compiled the same way) on the blocks stored in ref_schur.npz; the u
                        form both on the D block alone and on the full BD / GK (nc > ncu).

* ref_fbou.npz       -- outputs of the reference's generated boundary kernels
                        application/FM/ns/fbou_ns{2,3}d.c (types 1 far field, 2 adiabatic wall,
                        4 prescribed pressure) and application/FM/euler/fbou_euler{2,3}d.c (type 2
                        slip wall), and of the Roe matrices of application/FM/getan.c (absolute 0
                        and 1, with and without the entropy fix), on seeded random states; compiled
                        into oracle/_ref by oracle/build_ref.sh.

* binfile_format.json -- the header positions (ndims(k) = ...) and the fwrite sequence of the
                        single-process branch of util/writeBinaryFile.m, read from its source.

Usage: python tests/golden/make_golden.py REFERENCE_ROOT [--only adjoint|fbou|master|binfile]
       (or set HDG_REFERENCE)
"""
import os
import sys
from pathlib import Path

import numpy as np
import scipy.io as sio

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
OUT = Path(__file__).resolve().parent

MASTER_FIELDS = ["nd", "porder", "plocvl", "plocfc", "perm", "gpvl", "gwvl", "shapvl", "gpfc", "gwfc",
                 "shapfc", "shapvgdotshapvl", "shapvt", "shapvg", "shapfgdotshapfc", "shapft", "shapfg"]


def _master(struct):
    out = {}
    for k in MASTER_FIELDS:
        if k in struct.dtype.names:
            out[k] = np.array(struct[k], dtype=np.float64)
    return out


def adjoint_fixture():
    from oracle import oracle as O
    d = np.load(OUT / "ref_schur.npz")
    adj = {}
    for tag in ("euler2d", "ns2d"):
        g = lambda k: np.array(d[f"{tag}_{k}"])
        npv, ncu, _, nc, ne = g("BD").shape
        ndf = g("H").shape[1]
        outs = O.ref_mex("schur_uq_adjoint.so", [g(k) for k in ("M", "C", "E", "BD", "F", "GK", "H", "Rq", "Ru", "Rh")],
                         [(npv, nc, ne), (npv, nc, ncu, ndf, ne), (ncu, ndf, ncu, ndf, ne), (ncu, ndf, ne)])
        for k, v in zip(("DUDG", "DUDG_DUH", "AE", "FE"), outs):
            adj[f"{tag}_uqadj_{k}"] = v
        for form, BD, GK in (("uadj", g("BDu"), g("GKu")), ("uadjfull", g("BD"), g("GK"))):
            ncx = BD.shape[3]
            outs = O.ref_mex("schur_u_adjoint.so", [BD, g("F"), GK, g("H"), g("Ru"), g("Rh")],
                             [(npv, ncx, ne), (npv, ncx, ncu, ndf, ne), (ncu, ndf, ncu, ndf, ne), (ncu, ndf, ne)])
            for k, v in zip(("DUDG", "DUDG_DUH", "AE", "FE"), outs):
                adj[f"{tag}_{form}_{k}"] = v
    np.savez_compressed(OUT / "ref_schur_adjoint.npz", **adj)


def master_p4_fixture(ref):
    """Face tables of the p=4 master in problem/burgers/results.mat (a quadrilateral master, so
    only its 1D face tables are shared with the simplices)."""
    d = sio.loadmat(str(Path(ref) / "problem/burgers/results.mat"), struct_as_record=True)
    m = d["master"][0, 0]
    assert int(np.array(m["porder"]).ravel()[0]) == 4 and int(np.array(m["nd"]).ravel()[0]) == 2
    np.savez_compressed(OUT / "master_seg_p4.npz", **{k: np.array(m[k], dtype=np.float64)
                                                      for k in ("plocfc", "gpfc", "gwfc", "shapfc")})


def fbou_states(nd, ng, seed):
    """Seeded face-point states: interior udg[ng, nc], trace uh[ng, ncu], unit normals nl[ng, nd]
    (every other normal nearly perpendicular to the velocity, so that |un| < eps c there and the
    entropy fix of getan.m is exercised), a boundary state ub[ncu]."""
    rng = np.random.default_rng(seed)
    gam, minf = 1.4, 0.5
    ncu = nd + 2
    rho = 1.0 + 0.1 * rng.standard_normal(ng)
    vel = 0.3 * rng.standard_normal((ng, nd)) + np.eye(nd)[0]
    p = (1.0 + 0.05 * rng.standard_normal(ng)) / (gam * minf * minf)
    u = np.column_stack([rho, rho[:, None] * vel, p / (gam - 1) + 0.5 * rho * (vel ** 2).sum(1)])
    uh = u * (1.0 + 0.02 * rng.standard_normal(u.shape))
    q = 0.1 * rng.standard_normal((ng, ncu * nd))
    nl = rng.standard_normal((ng, nd))
    vh = uh[:, 1:nd + 1] / uh[:, :1]
    for g in range(0, ng, 2):                       # nearly tangential: un ~ 0
        nl[g] -= (nl[g] @ vh[g]) / (vh[g] @ vh[g]) * vh[g]
        nl[g] += 1e-3 * vh[g]
    nl /= np.linalg.norm(nl, axis=1)[:, None]
    ub = np.concatenate([[1.0], np.eye(nd)[0], [1.0 / (gam * (gam - 1) * minf * minf) + 0.5]])
    return np.column_stack([u, q]), uh, nl, ub


def fbou_fixture():
    import ctypes as ct
    from oracle import oracle as O
    v = lambda a: a.ctypes.data_as(ct.c_void_p)
    out = {}
    for fam, types in (("ns", (1, 2, 4)), ("euler", (2,))):
        L = ct.CDLL(str(O.HERE / "_ref" / f"libref_fbou_{fam}.so"))
        for nd in (2, 3):
            ncu, ng = nd + 2, 16
            nc = ncu * (nd + 1)
            udg, uh, nl, ub = (np.asfortranarray(a) for a in fbou_states(nd, ng, 7 + nd))
            pg = np.zeros((ng, nd), order="F")
            for eps in (0.0, 0.5):
                param = np.array([1.4, eps, 1000.0, 0.72, 0.5, 2.0])
                tag = f"{fam}{nd}d_e{int(eps > 0)}"
                out[tag + "_udg"], out[tag + "_uh"], out[tag + "_nl"], out[tag + "_ub"] = udg, uh, nl, ub
                out[tag + "_param"] = param
                for ib in types:
                    fh = np.zeros((ng, ncu), order="F"); fu = np.zeros((ng, ncu, nc), order="F")
                    fhh = np.zeros((ng, ncu, ncu), order="F")
                    L.ref_fbou(v(fh), v(fu), v(fhh), v(pg), v(udg), v(uh), v(nl), v(ub), v(param), ct.c_double(0.0),
                               ib, ng, ncu, nc, nd, nd)
                    out[f"{tag}_ib{ib}_fh"], out[f"{tag}_ib{ib}_fh_udg"], out[f"{tag}_ib{ib}_fh_uh"] = fh, fu, fhh
                if fam == "ns":
                    for ab in (0, 1):
                        An = np.zeros((ng, ncu, ncu), order="F"); Anm = np.zeros((ng, ncu, ncu, ncu), order="F")
                        L.ref_getan(v(An), v(Anm), v(uh), v(nl), v(param), ab, ng, ncu, nd)
                        out[f"{tag}_getan{ab}_An"], out[f"{tag}_getan{ab}_Anm"] = An, Anm
    np.savez_compressed(OUT / "ref_fbou.npz", **out)


def binfile_fixture(ref):
    import json
    import re
    src = (Path(ref) / "util/writeBinaryFile.m").read_text()
    start = src.index("if nproc == 1")
    block = src[start:src.index("fclose(fileID);", start)]
    code = "\n".join(line.split("%")[0] for line in block.splitlines())
    header = {int(k): v.strip() for k, v in re.findall(r"ndims\((\d+)\)\s*=\s*([^;]+);", code)}
    fwrites = [v.strip() for v in re.findall(r"fwrite\(fileID,\s*([^,]+),'double',endian\);", code)]
    (OUT / "binfile_format.json").write_text(json.dumps({"header": header, "fwrites": fwrites}, indent=1) + "\n")


def main(ref):
    ref = Path(ref)
    from oracle import oracle as O
    from hdg_b200 import configs

    d = sio.loadmat(ref / "master/testpython.mat")
    np.savez_compressed(OUT / "master_tri_p2.npz", **_master(d["masterm"][0, 0]))

    rng = np.random.default_rng(20261203)
    phys = {}
    for nd in (2, 3):
        ncu = nd + 2; nc = ncu * (nd + 1); ng = 40
        udg = 0.05 * rng.standard_normal((ng, nc))
        udg[:, 0] = 1.0 + 0.1 * rng.random(ng)
        udg[:, 1:nd + 1] = rng.standard_normal((ng, nd))
        udg[:, ncu - 1] = 5.0 + rng.random(ng)
        nl = rng.standard_normal((ng, nd)); nl /= np.linalg.norm(nl, axis=1, keepdims=True)
        uh = udg[:, :ncu] + 0.01 * rng.standard_normal((ng, ncu))
        for tag, param in (("ns", [1.4, 0.0, 1000.0, 0.72, 0.3, 2.0]), ("euler", [1.4, 0.0, np.inf, 0.72, 0.5, 2.0])):
            param = np.array(param)
            # Euler: application/FM/euler kernels on the u-only state (nc = ncu)
            src = udg if tag == "ns" else np.asfortranarray(udg[:, :ncu])
            f, fu = O.ref_flux(nd, param, src, tag)
            fh, fhu, fhh = O.ref_fhat(nd, param, nl, src, uh, tag)
            p = f"{tag}{nd}d_"
            phys.update({p + "param": param, p + "udg": udg, p + "nl": nl, p + "uh": uh, p + "f": f,
                         p + "f_udg": fu, p + "fh": fh, p + "fh_udg": fhu, p + "fh_uh": fhh})
    np.savez_compressed(OUT / "ref_physics.npz", **phys)

    sch = {}
    for tag, P in (("euler2d", configs.c1(n=2, porder=2)), ("ns2d", configs.c2(n=1, porder=3))):
        m, a = P.master, P.app
        blk = O.hdg_elemental(m, a, P.mesh.dgnodes, P.mesh.bf, P.UDG, P.uh_elem(), P.SH, intermediates=True)
        ne = P.mesh.ne; npv = m.npv; nc = a.nc; ncu = a.ncu; ndf = m.npf * m.nfe
        keys = ("M", "C", "E", "BD", "F", "GK", "H", "Rq", "Ru", "Rh")
        outs = O.ref_mex("schur_uq.so", [blk[k].copy() for k in keys],
                         [(npv, nc, ne), (npv, nc, ncu, ndf, ne), (ncu, ndf, ncu, ndf, ne), (ncu, ndf, ne)])
        for k in keys:
            sch[f"{tag}_{k}"] = blk[k]
        for k, v in zip(("DUDG", "DUDG_DUH", "AE", "FE"), outs):
            sch[f"{tag}_uq_{k}"] = v
        # u-only form: D block and the u columns of GK
        BDu = np.asfortranarray(blk["BD"][:, :, :, :ncu, :])
        GKu = np.asfortranarray(blk["GK"][:, :, :, :ncu, :])
        outs = O.ref_mex("schur_u.so", [BDu, blk["F"].copy(), GKu, blk["H"].copy(), blk["Ru"].copy(), blk["Rh"].copy()],
                         [(npv, ncu, ne), (npv, ncu, ncu, ndf, ne), (ncu, ndf, ncu, ndf, ne), (ncu, ndf, ne)])
        sch[f"{tag}_BDu"] = BDu
        sch[f"{tag}_GKu"] = GKu
        for k, v in zip(("DUDG", "DUDG_DUH", "AE", "FE"), outs):
            sch[f"{tag}_u_{k}"] = v
    np.savez_compressed(OUT / "ref_schur.npz", **sch)
    adjoint_fixture()
    fbou_fixture()
    master_p4_fixture(ref)
    binfile_fixture(ref)
    for f in sorted(OUT.glob("*.npz")):
        print(f.name, f.stat().st_size)


def reference_root(args):
    """The reference tree: the first argument, else $HDG_REFERENCE."""
    root = args[0] if args else os.environ.get("HDG_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT [--only adjoint|binfile] (or set HDG_REFERENCE)")
    return root


if __name__ == "__main__":
    args = [x for x in sys.argv[1:] if not x.startswith("--only")]
    only = sys.argv[sys.argv.index("--only") + 1] if "--only" in sys.argv else None
    args = [x for x in args if x != only]
    if only == "adjoint":
        adjoint_fixture()
    elif only == "fbou":
        fbou_fixture()
    elif only == "master":
        master_p4_fixture(reference_root(args))
    elif only == "binfile":
        binfile_fixture(reference_root(args))
    else:
        main(reference_root(args))
