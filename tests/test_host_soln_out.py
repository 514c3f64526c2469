"""Host logic of exf_write_xdmf (no GPU): the solution output of print_soln written as
XDMF over binary datasets, checked against the reference's own tables (the Quad9 / Hex27
split into linear sub-cells of MGMesh::print_conn_lin_hf5 and the element map Prol of
MGGeomEl, tests/golden/mggeomel.json) on refined meshes, and read back."""
import json
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import exfemus_b200 as ex
from exfemus_b200 import _lib

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mggeomel.json")))


def table(key, dtype=float):
    t = GOLD[key]
    return np.array(t["data"], dtype=dtype).reshape(t["shape"])


def top_mesh(dim, nlev):
    """The top level of a refined skewed box: xyz [dim][n], conn [nel][9 | 27]."""
    if dim == 2:
        xyz0 = np.array([[0, 2, 2.5, 0.3, 1, 2.2, 1.4, 0.15, 1.2], [0, 0.2, 1.6, 1, 0.1, 0.9, 1.3, 0.5, 0.7]])
        conn0 = np.arange(9)[None, :]
        nv = 4
    else:
        xyz0 = unit_hex27()
        xyz0 = xyz0 + 0.1 * np.sin(3.0 * xyz0[::-1])  # a curved hex27
        conn0, nv = np.arange(27)[None, :], 8
    r = ex.Mesh.refine_arrays(dim, nlev, nv, xyz0, conn0)
    return r["xyz"], r["conn"][nlev - 1]


def unit_hex27():
    """Coordinates [3][27] of one hex27 element on [0,2]^3 in libMesh local order: each
    node at its offset in half-element units (vertices, edges, faces, centre)."""
    from itertools import product
    pts = [(0, 0, 0), (2, 0, 0), (2, 2, 0), (0, 2, 0), (0, 0, 2), (2, 0, 2), (2, 2, 2), (0, 2, 2),
           (1, 0, 0), (2, 1, 0), (1, 2, 0), (0, 1, 0), (0, 0, 1), (2, 0, 1), (2, 2, 1), (0, 2, 1),
           (1, 0, 2), (2, 1, 2), (1, 2, 2), (0, 1, 2),
           (1, 1, 0), (1, 0, 1), (2, 1, 1), (1, 2, 1), (0, 1, 1), (1, 1, 2), (1, 1, 1)]
    assert set(pts) == set(product(range(3), repeat=3))
    return np.array(pts, float).T


@pytest.mark.parametrize("dim,nlev", [(2, 3), (3, 2)])
def test_subcells_coordinates_and_fields(tmp_path, dim, nlev):
    xyz, conn = top_mesh(dim, nlev)
    nn = xyz.shape[1]
    nvx = 4 if dim == 2 else 8
    rng = np.random.default_rng(dim)
    u = rng.standard_normal(nn)
    p = np.full(nn, np.nan)  # a linear variable: only the element vertices are read
    vx = np.unique(conn[:, :nvx])
    p[vx] = rng.standard_normal(vx.size)
    path = ex.write_xdmf(dim, xyz, conn, [("u", 2, u), ("p", 1, p)], t_step=7, time=0.35,
                         out_dir=str(tmp_path), ndigits=3)
    assert os.path.basename(path) == "sol.007.xmf"
    assert sorted(os.listdir(tmp_path)) == ["mesh.007.bin", "mesh_conn_lin.bin", "sol.007.bin", "sol.007.xmf"]
    d = ex.read_xdmf(path)
    assert d["time"] == 0.35
    assert d["cell_type"] == ("Quadrilateral" if dim == 2 else "Hexahedron")
    # MSH0CONN: the reference's sub-cell table applied element by element
    lin = table("quad9_conn_lin" if dim == 2 else "hex27_conn_lin", int)
    assert np.array_equal(d["cells"], conn[:, lin].reshape(-1, nvx))
    # X1, X2, X3
    assert np.array_equal(d["xyz"][:dim], xyz)
    assert d["xyz"].shape == (3, nn) and (dim == 3 or not d["xyz"][2].any())
    # the quadratic variable as given, the linear one by the reference's Prol, summed by vertex
    assert np.array_equal(d["fields"]["u"], u)
    P = table("quad9_prol" if dim == 2 else "hex27_prol")
    want = np.zeros(nn)
    for c in conn:
        for k in range(conn.shape[1]):
            s = 0.0
            for j in range(nvx):
                s += P[k, j] * p[c[j]]
            want[c[k]] = s
    assert np.array_equal(d["fields"]["p"], want)
    assert np.array_equal(d["fields"]["p"][vx], p[vx])


def test_xdmf_text(tmp_path):
    xyz, conn = top_mesh(2, 2)
    nn = xyz.shape[1]
    path = ex.write_xdmf(2, xyz, conn, [("T", 2, np.arange(nn, dtype=float))], t_step=12, time=1.5,
                         out_dir=str(tmp_path), basesol="run", basemesh="grid", connlin="_lin")
    root = ET.parse(path).getroot()
    grid = root.find("Domain").find("Grid")
    assert grid.get("Name") == "Mesh"
    topo = grid.find("Topology")
    assert topo.get("Dimensions") == str(conn.shape[0] * 4)
    ds = topo.find("DataStructure")
    assert ds.text.strip() == "grid_lin.bin" and ds.get("Format") == "Binary" and ds.get("Seek") == "0"
    geo = grid.find("Geometry")
    assert geo.get("Type") == "X_Y_Z"
    assert [g.get("Seek") for g in geo.findall("DataStructure")] == [str(k * nn * 8) for k in range(3)]
    assert all(g.text.strip() == "grid.0012.bin" for g in geo.findall("DataStructure"))
    (att,) = grid.findall("Attribute")
    assert att.get("Name") == "T" and att.get("Center") == "Node"
    assert att.find("DataItem").text.strip() == "run.0012.bin"
    assert os.path.getsize(os.path.join(tmp_path, "run.0012.bin")) == nn * 8


def test_bad_output_arguments(tmp_path):
    xyz, conn = top_mesh(2, 2)
    nn = xyz.shape[1]
    with pytest.raises(_lib.ExfError) as e:
        ex.write_xdmf(2, xyz, conn, [("u", 3, np.zeros(nn))], out_dir=str(tmp_path))
    assert e.value.code == _lib.EXF_ERR_ARG
    with pytest.raises(_lib.ExfError) as e:
        ex.write_xdmf(2, xyz, conn, [('a"b', 2, np.zeros(nn))], out_dir=str(tmp_path))
    assert e.value.code == _lib.EXF_ERR_ARG
    bad = conn.copy()
    bad[0, 3] = nn
    with pytest.raises(_lib.ExfError) as e:
        ex.write_xdmf(2, xyz, bad, [("u", 2, np.zeros(nn))], out_dir=str(tmp_path))
    assert e.value.code == _lib.EXF_ERR_ARG
    with pytest.raises(_lib.ExfError) as e:
        ex.write_xdmf(2, xyz, conn, [("u", 2, np.zeros(nn))], out_dir=str(tmp_path / "missing"))
    assert e.value.code == _lib.EXF_ERR_IO
    assert b"cannot open" in _lib.load().exf_last_error()


def test_case_file(tmp_path):
    """The case file of print_case_xmf (src/MGEquationsSystem.C:872-935): the base mesh
    coordinates <basemesh>.bin and no <Time>."""
    xyz, conn = top_mesh(3, 2)
    nn = xyz.shape[1]
    f = np.arange(nn, dtype=float)
    path = ex.write_xdmf(3, xyz, conn, [("T", 2, f), ("Tbd", 2, f % 2), ("Tvl", 2, f % 3)], t_step=0,
                         out_dir=str(tmp_path), basesol="case", basemesh="grid", case=True)
    assert os.path.basename(path) == "case.0000.xmf"
    assert sorted(os.listdir(tmp_path)) == ["case.0000.bin", "case.0000.xmf", "grid.bin", "grid_conn_lin.bin"]
    root = ET.parse(path).getroot()
    grid = root.find("Domain").find("Grid")
    assert grid.find("Time") is None
    assert all(g.text.strip() == "grid.bin" for g in grid.find("Geometry").findall("DataStructure"))
    d = ex.read_xdmf(path)
    assert d["time"] is None
    assert np.array_equal(d["xyz"], xyz)
    assert [a.get("Name") for a in grid.findall("Attribute")] == ["T", "Tbd", "Tvl"]
    assert np.array_equal(d["fields"]["Tvl"], f % 3)
