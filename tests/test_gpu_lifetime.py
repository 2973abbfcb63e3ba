"""Handle lifetimes across the C ABI: every object holds its context, so the
context handle may be destroyed first and the objects still work and free in
any order (as happens when a garbage collector finalises a reference cycle)."""
import numpy as np
import pytest

from delfem_b200 import meshes
from oracle import port as P

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def test_objects_outlive_their_context():
    from delfem_b200 import lib
    ctx = lib.Context(0)
    m = meshes.unit_square_tri(12)
    G = lib.Mesh(ctx, m.coord, m.elem)
    rp, ci = G.pattern()
    A = lib.Matrix(ctx, rp, ci, 1)
    b = torch.empty(m.nnode, dtype=torch.float64, device="cuda")
    G.assemble_poisson(A, 1.0, 1.0, b)
    fl = np.zeros(m.nnode, np.int32)
    fl[np.unique(m.bnd.ravel())] = 1
    lib.apply_dirichlet(A, torch.from_numpy(fl).cuda(), b)
    M = lib.ILU(A)
    M.factor()
    R = lib.RMatrix(ctx, 3, m.nnode, 1, 1, np.array([0, 1, 2, 3], np.uint32), np.array([0, 5, 9], np.uint32))
    ctx.close()  # the caller's handle goes first
    x = torch.zeros_like(b)
    r = b.clone()
    rc, it, conv = lib.solve_pcg(A, M, r, x, tol=1e-10, maxit=1000)
    assert rc == lib.OK and conv < 1e-10
    y = torch.empty_like(b)
    A.spmv(1.0, x, 0.0, y)
    torch.cuda.synchronize()
    assert float(torch.linalg.norm(y - b) / torch.linalg.norm(b)) < 1e-9
    # then the objects, in an order that frees the matrix before its ILU
    G.close()
    R.close()
    A.close()
    M.close()
    # the library still works on a fresh context
    ctx2 = lib.Context(0)
    S = P.System(rp, ci, 1)
    A2 = lib.Matrix(ctx2, rp, ci, 1)
    A2.set_values(np.full(S.N, 4.0), np.full(S.ncrs, -1.0))
    A2.close()
    ctx2.close()
