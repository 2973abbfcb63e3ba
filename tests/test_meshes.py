"""Synthetic mesh generators: the band numbering of the unit disk is a pure
renumbering of the ring numbering (same nodes, triangles and boundary bars,
same orientation) with an ILU(0) level depth of O(nring) instead of nnode."""
import numpy as np
import pytest

from delfem_b200 import meshes
from oracle import port as P


def _depth(m):
    rp, ci = P.pattern(m.nnode, m.elem)
    lev = np.zeros(m.nnode, np.int64)
    for i in range(m.nnode):
        c = ci[rp[i]:rp[i + 1]]
        c = c[c < i]
        lev[i] = lev[c].max() + 1 if c.size else 0
    return int(lev.max()) + 1


def _signed_area(m):
    p = m.coord[m.elem]
    return (p[:, 1, 0] - p[:, 0, 0]) * (p[:, 2, 1] - p[:, 0, 1]) - (p[:, 2, 0] - p[:, 0, 0]) * (p[:, 1, 1] - p[:, 0, 1])


@pytest.mark.parametrize("nring", [1, 5, 24])
def test_disk_band_numbering_is_a_renumbering(nring):
    a = meshes.unit_disk_tri(nring)
    b = meshes.unit_disk_tri(nring, numbering="bands")
    assert a.nnode == b.nnode and a.elem.shape == b.elem.shape and a.bnd.shape == b.bnd.shape
    # node correspondence by coordinates
    key = lambda c: [tuple(np.round(v, 12)) for v in c]
    pos = {k: i for i, k in enumerate(key(a.coord))}
    b2a = np.array([pos[k] for k in key(b.coord)])
    assert np.array_equal(np.sort(b2a), np.arange(a.nnode))
    tri = lambda e: sorted(tuple(np.roll(t, -int(np.argmin(t)))) for t in e)  # orientation-preserving
    assert tri(b2a[b.elem]) == tri(a.elem)
    bar = lambda e: sorted(tuple(sorted(t)) for t in e)
    assert bar(b2a[b.bnd]) == bar(a.bnd)
    assert (_signed_area(b) > 0).all()


def test_disk_level_depth():
    a = meshes.unit_disk_tri(30)
    b = meshes.unit_disk_tri(30, numbering="bands")
    assert _depth(a) == a.nnode  # ring numbering: one chain
    assert _depth(b) < 6 * 30
    with pytest.raises(ValueError):
        meshes.unit_disk_tri(3, numbering="spiral")


def test_sweep_partition_patches():
    """dfm_sweep_partition_patches (host only): every line of nodes along the
    box's long axis lies in one part; a square grid of patches across it."""
    from delfem_b200 import lib, meshes
    m = meshes.box_tet(20, 6, 6)
    part, nparts = lib.sweep_partition_patches(m.coord, 148)
    assert nparts == 144 or nparts <= 148
    p = part.reshape(7, 7, 21)  # nodes are x fastest: [k][j][i]
    assert (p == p[:, :, :1]).all()  # constant along x
    assert part.max() < nparts
    part2, n2 = lib.sweep_partition_patches(m.coord, 4)
    assert n2 == 4 and len(np.unique(part2)) == 4
    with pytest.raises(lib.DfmError):
        lib.sweep_partition_patches(m.coord, 0)
