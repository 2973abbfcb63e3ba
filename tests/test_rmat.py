"""Rectangular block-CRS matrices (MatVec::CMat_BlkCrs, the couplings between
segments of a linear system): the oracle's restatement of CMat_BlkCrs::MatVec
pinned bit for bit to the reference's own (oracle/_ref), every block shape
1..3 x 1..3, beta 0 and not; on the GPU, dfm_rmat_spmv against the oracle to
rounding (the device sums a row's blocks in lane order)."""
import numpy as np
import pytest

from oracle import port as P
from oracle import refshim as R

SHAPES = [(br, bc) for br in (1, 2, 3) for bc in (1, 2, 3)]


def _random_rmat(nrow, ncol, brow, bcol, seed):
    rng = np.random.default_rng(seed)
    rows = [np.sort(rng.choice(ncol, size=rng.integers(0, min(ncol, 6) + 1), replace=False)) for _ in range(nrow)]
    rp = np.concatenate([[0], np.cumsum([r.size for r in rows])]).astype(np.uint32)
    ci = np.concatenate(rows).astype(np.uint32) if rp[-1] else np.zeros(0, np.uint32)
    val = rng.standard_normal(int(rp[-1]) * brow * bcol)
    return rp, ci, val, rng.standard_normal(ncol * bcol), rng.standard_normal(nrow * brow)


@pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("brow,bcol", SHAPES)
def test_oracle_rmat_spmv_pinned_to_reference(brow, bcol):
    nrow, ncol = 57, 41
    rp, ci, val, x, y = _random_rmat(nrow, ncol, brow, bcol, 10 * brow + bcol)
    for alpha, beta in ((1.0, 0.0), (-1.0, 1.0), (0.7, -0.3)):
        ref = R.rmat_spmv(nrow, ncol, brow, bcol, rp, ci, val, alpha, x, beta, y)
        got = P.rmat_spmv(nrow, brow, bcol, rp, ci, val, alpha, x, beta, y)
        assert np.array_equal(got.view(np.uint64), ref.view(np.uint64)), (alpha, beta)


@pytest.mark.gpu
@pytest.mark.parametrize("brow,bcol", SHAPES)
def test_device_rmat_spmv_matches_oracle(ctx, brow, bcol):
    torch = pytest.importorskip("torch")
    from delfem_b200 import lib
    nrow, ncol = 3001, 1777
    rp, ci, val, x, y = _random_rmat(nrow, ncol, brow, bcol, 7 * brow + bcol)
    Rm = lib.RMatrix(ctx, nrow, ncol, brow, bcol, rp, ci)
    Rm.set_values(val)
    xd = torch.from_numpy(x).cuda()
    for alpha, beta in ((1.0, 0.0), (-1.0, 1.0), (0.7, -0.3)):
        yd = torch.from_numpy(y.copy()).cuda()
        Rm.spmv(alpha, xd, beta, yd)
        ctx.sync()
        ref = P.rmat_spmv(nrow, brow, bcol, rp, ci, val, alpha, x, beta, y)
        assert np.allclose(yd.cpu().numpy(), ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
    with pytest.raises(lib.DfmError):  # a column out of range
        lib.RMatrix(ctx, 2, 3, brow, bcol, np.array([0, 1, 2], np.uint32), np.array([0, 3], np.uint32))
    Rm.close()
