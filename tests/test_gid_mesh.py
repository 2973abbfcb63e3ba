"""The GiD ASCII mesh reader (dfm_gid_read_mesh, host only) against the
reference's own readers, Msh::CMesh3D::ReadFromFile_GiDMsh (tetrahedra,
hexahedra) and Msh::CMesher2D::ReadFromFile_GiDMsh (triangles given with
planar 3-D coordinates): the same coordinates, bit for bit, and the same
0-based connectivity; the pattern built from the read mesh is the reference's."""
import numpy as np
import pytest

from delfem_b200 import meshes
from oracle import port as P
from oracle import refshim as R
from tests import cases

needs_ref = pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) not present")


def _hexes(nx, ny, nz):
    mx, my = nx + 1, ny + 1
    idx = lambda a, b, c: a + mx * (b + my * c)  # noqa: E731
    h = []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                h.append([idx(i, j, k), idx(i + 1, j, k), idx(i + 1, j + 1, k), idx(i, j + 1, k),
                          idx(i, j, k + 1), idx(i + 1, j, k + 1), idx(i + 1, j + 1, k + 1), idx(i, j + 1, k + 1)])
    return np.array(h)


@needs_ref
def test_tetrahedra_match_reference(tmp_path):
    from delfem_b200 import lib
    m = meshes.box_tet(6, 3, 2)
    p = tmp_path / "box.msh"
    cases.write_gid_mesh(str(p), m.coord * np.pi, m.elem, "Tetrahedra")
    coord, elem = lib.read_gid_mesh(str(p))
    rc, rcoord, relem = R.gid_read(str(p), want2d=False)
    assert rc == 0
    assert np.array_equal(coord, rcoord) and np.array_equal(elem, relem)
    assert np.array_equal(elem, m.elem)
    # the pattern of the read mesh is the pattern of the mesh
    assert all(np.array_equal(a, b) for a, b in zip(P.pattern(coord.shape[0], elem), P.pattern(m.nnode, m.elem)))


@needs_ref
def test_hexahedra_match_reference(tmp_path):
    from delfem_b200 import lib
    m = meshes.box_tet(3, 2, 2)
    h = _hexes(3, 2, 2)
    p = tmp_path / "hex.msh"
    cases.write_gid_mesh(str(p), m.coord, h, "Hexahedra")
    coord, elem = lib.read_gid_mesh(str(p))
    rc, rcoord, relem = R.gid_read(str(p), want2d=False)
    assert rc == 0 and elem.shape == (12, 8)
    assert np.array_equal(coord, rcoord) and np.array_equal(elem, relem)


@needs_ref
@pytest.mark.parametrize("plane", ["xy", "yz", "zx"])
def test_planar_triangles_match_reference_2d_mesher(tmp_path, plane):
    """Triangles on a coordinate plane in 3-D: both readers drop the axis of
    least variance and keep the other two in cyclic order."""
    from delfem_b200 import lib
    m = meshes.unit_square_tri(5)
    u, v = m.coord[:, 0] * 1.7, m.coord[:, 1] * 0.9
    c3 = np.zeros((m.nnode, 3))
    a, b, z = {"xy": (0, 1, 2), "yz": (1, 2, 0), "zx": (2, 0, 1)}[plane]
    c3[:, a], c3[:, b], c3[:, z] = u, v, 0.25
    p = tmp_path / "tri.msh"
    cases.write_gid_mesh(str(p), c3, m.elem, "Triangle")
    coord, elem = lib.read_gid_mesh(str(p))
    rc, rcoord, relem = R.gid_read(str(p), want2d=True)
    assert rc == 0 and coord.shape == (m.nnode, 2)
    assert np.array_equal(coord, rcoord) and np.array_equal(elem, relem)
    assert np.array_equal(elem, m.elem)


def test_reader_matches_reference_fixture():
    """tests/golden/gid_*.msh as the reference's readers built them
    (tests/golden/make_golden.py)."""
    import os
    from delfem_b200 import lib
    g = os.path.join(os.path.dirname(__file__), "golden")
    ref = np.load(os.path.join(g, "gidref_meshes.npz"))
    coord, elem = lib.read_gid_mesh(os.path.join(g, "gid_box_tet.msh"))
    assert np.array_equal(coord, ref["tet_coord"]) and np.array_equal(elem, ref["tet_elem"])
    coord, elem = lib.read_gid_mesh(os.path.join(g, "gid_square_tri.msh"))
    assert np.array_equal(coord, ref["tri_coord"]) and np.array_equal(elem, ref["tri_elem"])


def test_two_d_file_and_rejections(tmp_path):
    from delfem_b200 import lib
    m = meshes.unit_square_tri(3)
    p = tmp_path / "tri2.msh"
    cases.write_gid_mesh(str(p), m.coord, m.elem, "Triangle", ndim=2)
    coord, elem = lib.read_gid_mesh(str(p))
    assert np.array_equal(coord, m.coord) and np.array_equal(elem, m.elem)
    # a non-planar triangle cloud (the reference's 2-D mesher refuses it too)
    c3 = np.hstack([m.coord, np.random.default_rng(0).random((m.nnode, 1))])
    cases.write_gid_mesh(str(p), c3, m.elem, "Triangle")
    with pytest.raises(lib.DfmError) as e:
        lib.read_gid_mesh(str(p))
    assert e.value.code == lib.ERR_INVALID
    if R.available():
        assert R.gid_read(str(p), want2d=True)[0] == 1
    bad = {
        "type": "MESH dimension 3 ElemType Prism Nnode 6\nCoordinates\nend coordinates\n\nElements\nend elements\n",
        "nnode": "MESH dimension 3 ElemType Tetrahedra Nnode 3\nCoordinates\n1 0 0 0\nend coordinates\n\n"
                 "Elements\nend elements\n",
        "node_range": "MESH dimension 3 ElemType Tetrahedra Nnode 4\nCoordinates\n1 0 0 0\n2 1 0 0\n3 0 1 0\n"
                      "4 0 0 1\nend coordinates\n\nElements\n1 1 2 3 5\nend elements\n",
        "ids": "MESH dimension 3 ElemType Tetrahedra Nnode 4\nCoordinates\n1 0 0 0\n3 1 0 0\nend coordinates\n\n"
               "Elements\nend elements\n",
        "truncated": "MESH dimension 3 ElemType Tetrahedra Nnode 4\nCoordinates\n1 0 0 0\n",
    }
    for name, text in bad.items():
        p.write_text(text)
        with pytest.raises(lib.DfmError) as e:
            lib.read_gid_mesh(str(p))
        assert e.value.code == lib.ERR_INVALID, name
    with pytest.raises(lib.DfmError) as e:
        lib.read_gid_mesh(str(tmp_path / "absent.msh"))
    assert e.value.code == lib.ERR_IO
