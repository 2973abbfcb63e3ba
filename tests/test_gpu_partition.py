"""Row partitions of the range-partitioned sweeps (dfm_ilu_set_sweep_partition):
the sweeps' results do not depend on which CTA takes which row, so every range
schedule with an arbitrary partition, and with the geometric patch partition,
matches the oracle as the natural ranges do."""
import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SYSTEMS = {
    "poisson_coef": lambda: cases.poisson(24, np.random.default_rng(3).lognormal(0, 1, 2 * 24 * 24))[1],
    "solid3d": lambda: cases.solid3d(8, 3, 3)[1],
    "random_b3": lambda: cases.random_spd_like(150, 3, 3),
    "helmholtz": lambda: cases.helmholtz(10)[1],
}


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()


def _make(ctx, S):
    from delfem_b200 import lib
    A = lib.Matrix(ctx, S.rowptr, S.colind, S.b, lib.COMPLEX if S.cplx else lib.REAL)
    A.set_values(S.diag, S.off)
    M = lib.ILU(A)
    M.factor()
    return A, M


@pytest.mark.parametrize("name", list(SYSTEMS))
@pytest.mark.parametrize("sweep", [3, 4, 5, 6, 7, 8, 9, 10])
def test_random_partition_every_range_mode(ctx, name, sweep):
    S = SYSTEMS[name]()
    A, M = _make(ctx, S)
    nparts = 7
    part = np.random.default_rng(sweep).integers(0, nparts, S.N).astype(np.uint32)
    M.set_sweep_partition(part, nparts)
    M.sweep = sweep
    _, fd, fo = S.ilu0()
    r = np.random.default_rng(11).standard_normal(S.N * S.xw)
    ref = S.precond(fd, fo, r)
    z = torch.zeros(S.N * S.xw, dtype=torch.float64, device="cuda")
    M.apply(_dev(r), z)
    got = z.cpu().numpy()
    assert np.allclose(got, ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())


def test_patch_partition_pcg(ctx):
    """The geometric patch partition of a box mesh, autotuned against the
    natural ranges: PCG to the oracle's x (the fused dots run over the
    partitioned slices too)."""
    from delfem_b200 import lib, meshes
    m, S = cases.solid3d(12, 4, 4)
    A, M = _make(ctx, S)
    part, nparts = lib.sweep_partition_patches(m.coord, 16)
    assert nparts <= 16
    M.set_sweep_partition(part, nparts)
    _, fd, fo = S.ilu0()
    ref = S.solve(fd, fo, method="pcg", tol=1e-10, maxit=2000)
    for sweep in (0, 3, 8, 9, 10):
        if sweep:
            M.sweep = sweep
        r = _dev(S.rhs)
        x = torch.zeros_like(r)
        rc, it, conv = lib.solve_pcg(A, M, r, x, tol=1e-10, maxit=2000)
        assert rc == lib.OK
        assert abs(it - ref["iters"]) <= 2
        xr = ref["x"]
        assert np.linalg.norm(x.cpu().numpy() - xr) <= 1e-8 * np.linalg.norm(xr)
    M.set_sweep_partition(None)  # back to the natural order
    r = _dev(S.rhs)
    x = torch.zeros_like(r)
    rc, it, conv = lib.solve_pcg(A, M, r, x, tol=1e-10, maxit=2000)
    assert rc == lib.OK and np.linalg.norm(x.cpu().numpy() - ref["x"]) <= 1e-8 * np.linalg.norm(ref["x"])


def test_partition_rejected(ctx):
    from delfem_b200 import lib
    S = SYSTEMS["poisson_coef"]()
    A, M = _make(ctx, S)
    with pytest.raises(lib.DfmError):
        M.set_sweep_partition(np.full(S.N, 3, np.uint32), 3)  # part index out of range
    with pytest.raises(lib.DfmError):
        M.set_sweep_partition(np.zeros(S.N, np.uint32), 100000)  # more parts than co-resident CTAs


@pytest.mark.parametrize("sweep", [0, 3, 7, 9, 10])
def test_partition_with_fill(ctx, sweep):
    """ILU(1) under the patch partition: the partition applies to the rows of
    the filled factor's pattern the same way; PCG to the oracle's x."""
    from delfem_b200 import lib
    m, S = cases.solid3d(12, 4, 4)
    A = lib.Matrix(ctx, S.rowptr, S.colind, S.b)
    A.set_values(S.diag, S.off)
    M = lib.ILU(A, fill_level=1)
    M.factor()
    M.set_sweep_partition(*lib.sweep_partition_patches(m.coord, 16))
    if sweep:
        M.sweep = sweep
    ns, fpat, fd, fo = S.iluk(1)
    ref = S.solve_fill(fpat, fd, fo, tol=1e-10, maxit=2000)
    r = _dev(S.rhs)
    x = torch.zeros_like(r)
    rc, it, conv = lib.solve_pcg(A, M, r, x, tol=1e-10, maxit=2000)
    assert rc == lib.OK and abs(it - ref["iters"]) <= 2
    assert np.linalg.norm(x.cpu().numpy() - ref["x"]) <= 1e-8 * np.linalg.norm(ref["x"])
