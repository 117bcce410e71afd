"""The on-disk state of util/writeBinaryFile.m (hdg_b200.binfile).

* The header positions and the order of the arrays equal those of writeBinaryFile.m's
  single-process branch, read from its source into tests/golden/binfile_format.json.
* write -> read round trips every array bit for bit, in all three byte orders, and the file is
  exactly the header plus the arrays (no padding, no missing values).
* The header describes the problem (sizes of the mesh, master, app and the block-CSR pattern)."""
import json
from pathlib import Path

import numpy as np
import pytest

from hdg_b200 import configs
from hdg_b200.binfile import FIELDS, HEADER, read_binary_file, state_arrays, write_binary_file

G = Path(__file__).resolve().parent / "golden"


def test_layout_follows_the_reference_writer():
    ref = json.loads((G / "binfile_format.json").read_text())
    assert {int(k): v for k, v in ref["header"].items()} == HEADER
    assert ref["fwrites"] == FIELDS


@pytest.mark.parametrize("endian", ["native", "ieee-le", "ieee-be"])
@pytest.mark.parametrize("name,kw", [("c1", dict(n=3, porder=2)), ("c4", dict(n=1, porder=2))])
def test_round_trip(tmp_path, endian, name, kw):
    P = configs.by_name(name, **kw)
    h, arrays = state_arrays(P.mesh, P.master, P.app, P.UDG, P.UH)
    path = write_binary_file(tmp_path / "state", P.mesh, P.master, P.app, P.UDG, P.UH, endian=endian)
    assert path.stat().st_size == 8 * sum(a.size for a in arrays.values())
    st = read_binary_file(tmp_path / "state", endian=endian)
    assert st.header == {k: h[k] for k in HEADER.values()}
    assert list(st.arrays) == [f for f in FIELDS if f != "PDG"]
    for k, a in arrays.items():
        assert np.array_equal(st.arrays[k], a), k
    assert np.array_equal(st.arrays["UDG"], P.UDG) and np.array_equal(st.arrays["UH"], P.UH)
    assert np.array_equal(st.arrays["mesh.t2f"], P.mesh.t2f)
    if endian != "native":
        other = "ieee-be" if endian == "ieee-le" else "ieee-le"
        with pytest.raises(ValueError):
            read_binary_file(tmp_path / "state", endian=other)      # sizes decode as garbage


def test_header_describes_the_problem():
    P = configs.c2(n=3, porder=3)
    h, arrays = state_arrays(P.mesh, P.master, P.app, P.UDG, P.UH)
    m, mesh = P.master, P.mesh
    assert (h["mesh.nd"], h["mesh.ne"], h["mesh.nfe"]) == (2, mesh.t2f.shape[0], 3)
    assert (h["master.npe"], h["master.npf"], h["master.nge"], h["master.ngf"]) == (10, 4, 12, 4)
    assert (h["app.nc"], h["app.ncu"], h["app.nch"], h["app.ncq"]) == (12, 4, 4, 8)
    assert h["mesh.cbsr_nblks"] == int(mesh.cbsr_rowpts[-1]) == np.asarray(mesh.cbsr_colind).size
    assert h["mesh.blkSize"] == 16 and h["mesh.ndh"] == P.UH.shape[1] == h["mesh.nf"] * 4
    assert arrays["ndims"][39] == 1.0                                  # nproc


def test_truncated_file_is_rejected(tmp_path):
    P = configs.c1(n=2, porder=1)
    path = write_binary_file(tmp_path / "s", P.mesh, P.master, P.app, P.UDG, P.UH)
    raw = path.read_bytes()
    (tmp_path / "t.bin").write_bytes(raw[:-8])
    with pytest.raises(ValueError):
        read_binary_file(tmp_path / "t")
