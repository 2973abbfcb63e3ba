"""dfm_ilu_apply_static, the allocation-free preconditioner application.

It exists for callers that cannot allocate device memory where they apply the
preconditioner (code that enqueues work on a stream it must not stall,
frameworks that own every device allocation, callbacks under an allocator
lock): it keeps its intermediate vector in a static device array instead, and
only enqueues its sweeps.  These tests call it through the C ABI, twice in a
row per system, and compare it with the existing entry point dfm_ilu_apply at
the tolerance the other sweep tests use, and with the oracle's ILU(0)
application (forward + backward substitution of the reference's factor).  The
file is named to be collected last and creates its own context, so it runs the
same alone or after the rest.
"""
import ctypes

import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

MAX_DOUBLES = 1 << 19  # size of the static scratch array (4 MiB)
RTOL = 1e-11           # the sweep tests' tolerance (summation order differs)


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float64)).cuda()


@pytest.fixture(scope="module")
def nctx():
    from delfem_b200 import lib
    c = lib.Context(0)
    yield c
    c.close()


SYSTEMS = {
    "poisson48": lambda: cases.poisson(48)[1],
    "solid2d": lambda: cases.solid2d(10, np.random.default_rng(2).lognormal(0, 0.5, 200))[1],
    "solid3d": lambda: cases.solid3d(6, 2, 2)[1],
    "helmholtz": lambda: cases.helmholtz(8)[1],
}


def _close(got, ref):
    return np.allclose(got, ref, rtol=RTOL, atol=RTOL * np.abs(ref).max())


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_static_apply_matches_apply_twice(nctx, name):
    from delfem_b200 import lib
    S = SYSTEMS[name]()
    ns, fd, fo = S.ilu0()
    A = lib.Matrix(nctx, S.rowptr, S.colind, S.b, lib.COMPLEX if S.cplx else lib.REAL)
    A.set_values(S.diag, S.off)
    M = lib.ILU(A)
    M.factor()
    rng = np.random.default_rng(17)
    L = lib.lib()
    for call in range(2):  # two calls in a row share the static array
        rh = rng.standard_normal(S.N * S.xw)
        r = _dev(rh)
        z_ref = torch.zeros_like(r)
        M.apply(r, z_ref)
        z = torch.full_like(r, float("nan"))
        torch.cuda.synchronize()
        rc = L.dfm_ilu_apply_static(M.h, ctypes.c_void_p(r.data_ptr()), ctypes.c_void_p(z.data_ptr()))
        assert rc == lib.OK, (name, call, rc)
        nctx.sync()  # the call only enqueues its sweeps on the context's stream
        assert nctx.take_error() == (0, 0)
        got = z.cpu().numpy()
        assert _close(got, z_ref.cpu().numpy()), (name, call)
        assert _close(got, S.precond(fd, fo, rh)), (name, call)


def test_static_apply_rejects_systems_beyond_the_array(nctx):
    from delfem_b200 import lib
    N = MAX_DOUBLES + 1  # one scalar row too many
    rowptr = np.zeros(N + 1, np.uint32)
    A = lib.Matrix(nctx, rowptr, np.zeros(0, np.uint32), 1)
    A.set_values(np.ones(N), np.zeros(0))
    M = lib.ILU(A)
    M.factor()
    r = torch.ones(N, dtype=torch.float64, device="cuda")
    z = torch.zeros_like(r)
    torch.cuda.synchronize()
    rc = lib.lib().dfm_ilu_apply_static(M.h, ctypes.c_void_p(r.data_ptr()), ctypes.c_void_p(z.data_ptr()))
    assert rc == lib.ERR_INVALID
