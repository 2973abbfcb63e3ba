"""Boundary facets of GiD meshes (dfm_gid_boundary, host only) against what the
reference's own readers derive and store: Msh::CMesh3D::ReadFromFile_GiDMsh's
colour-coded boundary triangle arrays (tetrahedra) and
Msh::CMesher2D::ReadFromFile_GiDMsh's outer bar arrays and their end vertices
(triangles, quadrilaterals).  The same facets, node for node, in the same
groups and order; for 2-D the same vertices and chain ends.  Cases: clean
boxes, jittered nodes (many colours, normals near the threshold), random
subsets of elements (non-manifold edges and pinched nodes), an inverted
tetrahedron (the reference leaves its faces unlinked), quadrilaterals."""
import os

import numpy as np
import pytest

from delfem_b200 import meshes
from oracle import refshim as R
from tests import cases

needs_ref = pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) not present")


def _grouped(g):
    return np.concatenate([g["facets"][k] for k in g["groups"]]) if g["groups"] else g["facets"][:0]


def _check(g, r):
    assert len(g["groups"]) == len(r["groups"])
    assert [len(k) for k in g["groups"]] == [len(k) for k in r["groups"]]
    assert np.array_equal(_grouped(g), r["facets"])
    # every facet lands in exactly one group
    assert sorted(np.concatenate(g["groups"]).tolist() if g["groups"] else []) == list(range(g["facets"].shape[0]))
    assert np.array_equal(g["vertices"], r["vertices"])
    assert np.array_equal(g["ends"], r["ends"])
    # the reference numbers the element array 1, the groups 2.., the vertices after them
    assert list(r["group_ids"]) == list(range(2, 2 + len(r["groups"])))
    if len(r["vertices"]):
        assert list(r["vertex_ids"]) == list(range(2 + len(r["groups"]), 2 + len(r["groups"]) + len(r["vertices"])))


def _tet_case(tmp_path, coord, elem, name):
    from delfem_b200 import lib
    p = str(tmp_path / f"{name}.msh")
    cases.write_gid_mesh(p, coord, elem, "Tetrahedra")
    c, e = lib.read_gid_mesh(p)
    g = lib.gid_boundary(c, e)
    _check(g, R.gid_boundary(p, want2d=False))
    return g


def _planar_case(tmp_path, coord2, elem, name, kind="Triangle"):
    from delfem_b200 import lib
    c3 = np.zeros((coord2.shape[0], 3))
    c3[:, 1], c3[:, 2], c3[:, 0] = coord2[:, 0], coord2[:, 1], -0.5  # on the plane x = -0.5
    p = str(tmp_path / f"{name}.msh")
    cases.write_gid_mesh(p, c3, elem, kind)
    c, e = lib.read_gid_mesh(p)
    g = lib.gid_boundary(c, e)
    _check(g, R.gid_boundary(p, want2d=True))
    return g


@needs_ref
def test_box_faces_are_six_colours(tmp_path):
    m = meshes.box_tet(6, 3, 2)
    g = _tet_case(tmp_path, m.coord * np.pi, m.elem, "box")
    assert len(g["groups"]) == 6
    assert g["facets"].shape[0] == 2 * 2 * (6 * 3 + 3 * 2 + 6 * 2)


@needs_ref
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_jittered_box_matches_reference(tmp_path, seed):
    m = meshes.box_tet(5, 4, 3)
    rng = np.random.default_rng(seed)
    g = _tet_case(tmp_path, m.coord + 0.08 * rng.standard_normal(m.coord.shape), m.elem, f"jit{seed}")
    assert len(g["groups"]) > 6


@needs_ref
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_tet_subsets_non_manifold_match_reference(tmp_path, seed):
    rng = np.random.default_rng(seed)
    m = meshes.box_tet(5, 4, 3)
    keep = rng.random(m.elem.shape[0]) < 0.6
    _tet_case(tmp_path, m.coord * 1.1 + 0.02 * rng.standard_normal(m.coord.shape), m.elem[keep], f"sub{seed}")


@needs_ref
def test_inverted_tetrahedron_matches_reference(tmp_path):
    m = meshes.box_tet(3, 3, 3)
    e = m.elem.copy()
    e[40, [0, 1]] = e[40, [1, 0]]
    g = _tet_case(tmp_path, m.coord, e, "inv")
    assert g["facets"].shape[0] == 2 * 2 * 3 * 9 + 8  # its four faces and their partners' stay open


@needs_ref
def test_square_and_disk_chains(tmp_path):
    t = meshes.unit_square_tri(5)
    g = _planar_case(tmp_path, t.coord * np.array([1.7, 0.9]), t.elem, "square")
    assert len(g["groups"]) == 4 and len(g["vertices"]) == 4
    d = meshes.unit_disk_tri(8)
    g = _planar_case(tmp_path, d.coord, d.elem, "disk")
    assert len(g["groups"]) == 1 and len(g["vertices"]) == 1  # one closed chain


@needs_ref
@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_triangle_subsets_match_reference(tmp_path, seed):
    rng = np.random.default_rng(seed)
    t = meshes.unit_square_tri(8)
    keep = rng.random(t.elem.shape[0]) < 0.7
    _planar_case(tmp_path, t.coord + 0.01 * rng.standard_normal(t.coord.shape), t.elem[keep], f"tsub{seed}")


@needs_ref
def test_quadrilaterals_match_reference(tmp_path):
    nx, ny = 5, 3
    idx = lambda i, j: i + (nx + 1) * j  # noqa: E731
    q = np.array([[idx(i, j), idx(i + 1, j), idx(i + 1, j + 1), idx(i, j + 1)] for j in range(ny) for i in range(nx)])
    c = np.array([[i * 0.3, j * 0.5] for j in range(ny + 1) for i in range(nx + 1)])
    g = _planar_case(tmp_path, c, q, "quad", "Quadrilateral")
    assert len(g["groups"]) == 4 and g["facets"].shape[0] == 2 * (nx + ny)


def test_boundary_matches_reference_fixture():
    """tests/golden/gid_*.msh: the facets the reference's readers derived
    (tests/golden/make_golden.py)."""
    from delfem_b200 import lib
    gd = os.path.join(os.path.dirname(__file__), "golden")
    ref = np.load(os.path.join(gd, "gidref_meshes.npz"))
    for name, tag in (("gid_box_tet.msh", "tet"), ("gid_square_tri.msh", "tri")):
        c, e = lib.read_gid_mesh(os.path.join(gd, name))
        g = lib.gid_boundary(c, e)
        assert np.array_equal(_grouped(g), ref[f"{tag}_bnd_facets"])
        assert np.array_equal(np.cumsum([0] + [len(k) for k in g["groups"]]), ref[f"{tag}_bnd_group_ptr"])
        assert np.array_equal(g["vertices"], ref[f"{tag}_bnd_vertices"])
        assert np.array_equal(g["ends"].reshape(-1), ref[f"{tag}_bnd_ends"].reshape(-1))


def test_hexahedra_and_rejections():
    from delfem_b200 import lib
    c = np.random.default_rng(0).random((8, 3))
    g = lib.gid_boundary(c, np.arange(8)[None, :])
    assert g["facets"].shape[0] == 0 and not g["groups"]  # the reference derives no hexahedral boundary
    m = meshes.box_tet(2, 1, 1)
    e = m.elem.copy()
    e[0, 1] = e[0, 0]  # a repeated node
    with pytest.raises(lib.DfmError) as x:
        lib.gid_boundary(m.coord, e)
    assert x.value.code == lib.ERR_INVALID
    e = m.elem.copy()
    e[0, 2] = m.nnode  # out of range
    with pytest.raises(lib.DfmError):
        lib.gid_boundary(m.coord, e)
    with pytest.raises(lib.DfmError):  # prisms are no GiD element the readers take
        lib.gid_boundary(m.coord, np.zeros((1, 6), np.int32))
    # an empty mesh has no boundary
    g = lib.gid_boundary(m.coord, np.zeros((0, 4), np.int32))
    assert g["facets"].shape == (0, 3) and not g["groups"]
