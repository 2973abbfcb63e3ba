"""CLinearSystem_Save's stored boundary matrix (dfm_boundary_matrix, host
only) against the reference's own CMat_BlkCrs (SetPatternBoundary over K, the
two BC masks of FinalizeMarge, MatVec for MakeResidual): the same entries and
values bit for bit, and r = Force - B u to rounding; on the GPU the residual
through dfm_spmv."""
import numpy as np
import pytest

from oracle import port as P
from oracle import refshim as R
from tests import cases

needs_ref = pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) not present")


def _systems():
    """K before the Dirichlet elimination, its flags (clamped faces plus a few
    random DOFs, so that blocks are partly fixed) and prescribed values u."""
    rng = np.random.default_rng(4)
    out = []
    for name, (m, S), b in [("solid3d", cases.solid3d_raw(6, 2, 2), 3), ("solid2d", cases.solid2d_raw(6), 2),
                            ("poisson", cases.poisson_raw(8), 1)]:
        flags = P.bc_flags_from_bnd(m.nnode, b, m.bnd).astype(np.int32)
        extra = rng.random(flags.size) < 0.1
        flags[extra] = 1
        u = rng.standard_normal(flags.size)
        force = rng.standard_normal(flags.size)
        out.append((name, S, b, flags, u, force))
    return out


def _ref_B_in_our_layout(S, b, brow, bcol, bval):
    """The reference's rows (diagonal block first) as (diag, {col: block})."""
    N = S.N
    bb = b * b
    rows = []
    for i in range(N):
        ent = {}
        for k in range(brow[i], brow[i + 1]):
            ent[int(bcol[k])] = bval[k * bb:(k + 1) * bb]
        rows.append(ent)
    return rows


@needs_ref
@pytest.mark.parametrize("case", range(3))
def test_boundary_matrix_matches_reference(case):
    from delfem_b200 import lib
    name, S, b, flags, u, force = _systems()[case]
    brow, bcol, bdiag, boff = lib.boundary_matrix(S.rowptr, S.colind, S.diag, S.off, flags, b)
    rbrow, rbcol, rbval, rr = R.boundary_residual(S.N, b, S.rowptr, S.colind, S.diag, S.off, flags, force, u)
    ref = _ref_B_in_our_layout(S, b, rbrow, rbcol, rbval)
    bb = b * b
    for i in range(S.N):
        mine = {int(bcol[k]): boff[k * bb:(k + 1) * bb] for k in range(brow[i], brow[i + 1])}
        d = ref[i].pop(i, np.zeros(bb))
        assert np.array_equal(bdiag[i * bb:(i + 1) * bb], d), (name, i)
        assert mine.keys() == ref[i].keys(), (name, i)  # the same off-diagonal entries
        for j in mine:
            assert np.array_equal(mine[j], ref[i][j]), (name, i, j)
    # MakeResidual: the same product up to summation order
    Bs = P.System(brow, bcol, b)
    Bs.diag[:] = bdiag
    Bs.off[:] = boff
    r = Bs.spmv(-1.0, u, 1.0, force)
    assert np.allclose(r, rr, rtol=1e-13, atol=1e-13 * np.abs(rr).max())
    # and it is Force - K[:, fixed] u on the free rows, Force on the fixed ones
    Ks = P.System(S.rowptr, S.colind, b)
    Ks.diag[:] = S.diag
    Ks.off[:] = S.off
    ku = Ks.spmv(1.0, np.where(flags != 0, u, 0.0), 0.0, np.zeros_like(u))
    expect = np.where(flags == 0, force - ku, force)
    assert np.allclose(r, expect, rtol=1e-12, atol=1e-12 * np.abs(expect).max())


def test_boundary_matrix_edge_cases():
    from delfem_b200 import lib
    name, S, b, flags, u, force = _systems()[2]
    # nothing fixed: B is empty; everything fixed: B is empty too (no free row)
    for f in (np.zeros_like(flags), np.ones_like(flags)):
        brow, bcol, bdiag, boff = lib.boundary_matrix(S.rowptr, S.colind, S.diag, S.off, f, b)
        assert brow[-1] == 0 and not bdiag.any()
    with pytest.raises(lib.DfmError):
        bad = S.colind.copy()
        bad[0] = S.N + 5
        lib.boundary_matrix(S.rowptr, bad, S.diag, S.off, flags, b)


@pytest.mark.gpu
def test_make_residual_on_device(ctx):
    """MakeResidual as the library runs it: B on the device, r = Force - B u by
    dfm_spmv (alpha -1, beta 1), against the oracle's product."""
    torch = pytest.importorskip("torch")
    from delfem_b200 import lib
    for name, S, b, flags, u, force in _systems():
        brow, bcol, bdiag, boff = lib.boundary_matrix(S.rowptr, S.colind, S.diag, S.off, flags, b)
        B = lib.Matrix(ctx, brow, bcol, b)
        B.set_values(bdiag, boff)
        r = torch.from_numpy(force.copy()).cuda()
        B.spmv(-1.0, torch.from_numpy(u).cuda(), 1.0, r)
        Bs = P.System(brow, bcol, b)
        Bs.diag[:] = bdiag
        Bs.off[:] = boff
        ref = Bs.spmv(-1.0, u, 1.0, force)
        assert np.allclose(r.cpu().numpy(), ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max()), name
