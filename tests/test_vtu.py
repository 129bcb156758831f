"""The VTK XML writer (sp_vtu_write) on host arrays: the .pvtu index names
its piece, the piece holds the reference's point and cell arrays
(micro/src/output.c:65-188), hexahedra in the hexa8 node order of
src/fem.c:324-362, values round-tripping through the ascii text."""
import ctypes as C
import xml.etree.ElementTree as ET

import numpy as np

import madmax_b200 as mb
from oracle import oracle as O


def arrays(root):
    out = {}
    for da in root.iter("DataArray"):
        out[da.get("Name")] = np.array(da.text.split(), dtype=float)
    return out


def test_vtu_layout_and_values(tmp_path):
    n = np.array([2, 3, 2], dtype=np.int32)
    ln = np.array([1.0, 1.5, 0.5])
    nn, ne = 3 * 4 * 3, 12
    rng = np.random.default_rng(4)
    u, res = rng.standard_normal(3 * nn), rng.standard_normal(3 * nn)
    se, st = rng.standard_normal(6 * ne), rng.standard_normal(6 * ne) * 1e6
    et = (np.arange(ne) % 2).astype(np.uint8)
    base = str(tmp_path / "rve")
    rc = mb.lib().sp_vtu_write(base.encode(), mb.ptr(n, mb._ip), mb.ptr(ln), mb.ptr(u), mb.ptr(res),
                               mb.ptr(et, mb._up), mb.ptr(se), mb.ptr(st))
    assert rc == 0, mb.last_error()
    p = ET.parse(base + ".pvtu").getroot()
    assert p.find(".//Piece").get("Source") == "rve_0.vtu"
    names = [d.get("Name") for d in p.iter("PDataArray")]
    assert names == ["Position", "connectivity", "offsets", "types", "displ", "residual", "part",
                     "strain", "stress", "elem_type"]
    v = ET.parse(base + "_0.vtu").getroot()
    piece = v.find(".//Piece")
    assert int(piece.get("NumberOfPoints")) == nn and int(piece.get("NumberOfCells")) == ne
    a = arrays(v)
    m = O.mesh(3, list(n + 1), list(ln))
    nod = np.zeros(8, dtype=np.int32)
    conn = a["connectivity"].reshape(ne, 8).astype(int)
    for e in range(ne):
        O.lib().orc_elem_nodes(C.byref(m), e, O.ptr(nod, O._ip))
        assert list(conn[e]) == list(nod)
    assert (a["types"] == 12).all() and list(a["offsets"]) == [8 * (e + 1) for e in range(ne)]
    pos = a["Position"].reshape(nn, 3)
    x = np.zeros(3)
    for i in range(nn):
        O.lib().orc_node_coord(C.byref(m), i, O.ptr(x))
        assert np.allclose(pos[i], x, rtol=1e-6, atol=1e-12)
    for key, ref in (("displ", u), ("residual", res), ("strain", se), ("stress", st)):
        assert np.allclose(a[key], ref, rtol=1e-8, atol=0)
    assert (a["elem_type"] == et).all() and (a["part"] == 0).all()


def test_vtu_rejects_bad_mesh(tmp_path):
    n = np.array([2, 0, 2], dtype=np.int32)
    ln = np.ones(3)
    assert mb.lib().sp_vtu_write(str(tmp_path / "x").encode(), mb.ptr(n, mb._ip), mb.ptr(ln),
                                 None, None, None, None, None) == mb.SP_ERR_ARG
