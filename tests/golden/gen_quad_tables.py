"""Regenerate ``_quad_tables.py`` from the reference's tabulated simplex rules.

The reference integrates on triangles and tetrahedra with fixed tabulated rules
(``master/gaussquad2d.m`` and ``master/gaussquad3d.m``; the 3D weights are divided
by 6 at ``master/gaussquad3d.m:1771``).  Element-level parity with the reference
needs the *same* rule, digit for digit, so the numbers are carried over as data.
This script parses the two MATLAB files and writes the tables for the degrees the
hot path uses (triangles ``pgauss`` 1..8, tetrahedra ``pgauss`` 1..6).

Usage: ``python tests/golden/gen_quad_tables.py <path-to-reference-root>`` (or set ``HDG_REFERENCE``);
it writes ``hdg_b200/_quad_tables.py``.
"""
import os
import re
import sys
from pathlib import Path


def _parse(path, dim, maxdeg):
    txt = Path(path).read_text()
    body = txt.split("switch pgauss", 1)[1]
    blocks = re.split(r"\n\s*case\s+", body)[1:]
    out = {}
    for blk in blocks:
        head, rest = blk.split("\n", 1)
        head = head.strip()
        if head.startswith("{"):
            degs = [int(v) for v in head.strip("{}").split(",")]
        else:
            try:
                degs = [int(head.split()[0])]
            except ValueError:
                continue
        mw = re.search(r"w\s*=\s*\[(.*?)\]", rest, re.S)
        mx = re.search(r"x\s*=\s*\[(.*?)\]", rest, re.S)
        if not (mw and mx) or min(degs) > maxdeg:
            continue
        num = r"[-+]?\d*\.\d+(?:[eE][-+]?\d+)?"
        w = [float(v) for v in re.findall(num, mw.group(1))]
        xs = [float(v) for v in re.findall(num, mx.group(1))]
        assert len(xs) == dim * len(w), (path, degs, len(xs), len(w))
        x = [xs[i * dim:(i + 1) * dim] for i in range(len(w))]
        for d in degs:
            if d <= maxdeg:
                out[d] = (x, w)
    return out


def main(ref_root):
    tri = _parse(Path(ref_root) / "master/gaussquad2d.m", 2, 8)
    tet = _parse(Path(ref_root) / "master/gaussquad3d.m", 3, 6)
    lines = [
        '"""Tabulated simplex quadrature rules (generated by gen_quad_tables.py; do not edit).',
        "",
        "TRI[pgauss] = (points[n][2], weights[n]) on the unit right triangle, weights sum 1/2.",
        "TET[pgauss] = (points[n][3], weights[n]) on the unit right tetrahedron; the weights",
        "are stored as tabulated (they sum to 1) and are divided by 6 by the caller, as the",
        "reference does.",
        '"""',
        "",
    ]
    for name, tab in (("TRI", tri), ("TET", tet)):
        lines.append(f"{name} = {{")
        for d in sorted(tab):
            x, w = tab[d]
            lines.append(f"    {d}: (")
            lines.append("        [" + ", ".join("[" + ", ".join(repr(c) for c in p) + "]" for p in x) + "],")
            lines.append("        [" + ", ".join(repr(v) for v in w) + "],")
            lines.append("    ),")
        lines.append("}")
        lines.append("")
    dst = Path(__file__).resolve().parents[2] / "hdg_b200" / "_quad_tables.py"
    dst.write_text("\n".join(lines))
    print("wrote", dst, "tri degrees", sorted(tri), "tet degrees", sorted(tet))


if __name__ == "__main__":
    if len(sys.argv) < 2 and not os.environ.get("HDG_REFERENCE"):
        sys.exit("usage: gen_quad_tables.py REFERENCE_ROOT (or set HDG_REFERENCE)")
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ["HDG_REFERENCE"])
