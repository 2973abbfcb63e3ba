"""The time-integration variants of the stored-matrix linear system
(Fem::Ls::CLinearSystem_SaveDiaM_Newmark, first order, and
CLinearSystem_SaveDiaM_NewmarkBeta, second order): the stored matrix with its
fixed rows zeroed (SetBoundaryCondition_Row), MakeResidual's predictor and
r = force - B t, and UpdateValueOfField.

The oracle's restatement is pinned to the reference's own classes run through
the shim (oracle/_ref), bit for bit; on the GPU, dfm_mat_zero_rows and
dfm_newmark_update are bit-identical to the oracle, and dfm_newmark_residual
agrees to rounding (the device SpMV sums in its own order)."""
import numpy as np
import pytest

from delfem_b200 import meshes
from oracle import port as P
from oracle import refshim as R
from tests import cases

DT, GAMMA, BETA = 0.013, 0.6, 0.3025


def _case(scheme, n=9, seed=0):
    m = meshes.unit_square_tri(n)  # all four sides fixed
    b = 1 if scheme == 1 else 2
    rng = np.random.default_rng(seed + scheme)
    u, v, a, x = (rng.standard_normal(m.nnode * b) for _ in range(4))
    params = [1.3, 0.7, 0.4] if scheme == 1 else [cases.LAM2_PS, cases.MYU2, 1.1, 0.2, -0.5]
    rp, ci = P.pattern(m.nnode, m.elem)
    return m, b, rp, ci, params, u, v, a, x


def _eq(x, y):
    return np.array_equal(np.asarray(x).view(np.uint64), np.asarray(y).view(np.uint64))


@pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("scheme", [1, 2])
def test_oracle_pinned_to_reference_newmark(scheme):
    m, b, rp, ci, params, u, v, a, x = _case(scheme)
    ref = R.newmark(scheme, m, params, DT, GAMMA, BETA, u, v, a if scheme == 2 else None, x, ci.size)
    fl = ref["flags"]
    assert fl.sum() > 0 and fl.sum() < fl.size
    # the stored matrix after FinalizeMarge: zero rows at fixed DOFs, nothing else touched
    bb = b * b
    bd, bo = ref["bdiag"].reshape(-1, b, b), ref["boff"].reshape(-1, b, b)
    for i in range(m.nnode):
        for d in range(b):
            if fl[i * b + d]:
                assert not bd[i, d].any() and not bo[rp[i]:rp[i + 1], d].any()
    zd, zo = P.mat_zero_rows(m.nnode, b, rp, fl, ref["bdiag"], ref["boff"])
    assert _eq(zd, ref["bdiag"]) and _eq(zo, ref["boff"])  # idempotent on the reference's matrix
    r, nrm = P.newmark_residual(m.nnode, b, rp, ci, ref["bdiag"], ref["boff"], scheme, DT, GAMMA, BETA,
                                ref["force"], u, v, a if scheme == 2 else None, fl)
    assert _eq(r, ref["r"]) and _eq(nrm, ref["norm"])
    xo, uo, vo, ao = P.newmark_update(scheme, DT, GAMMA, BETA, fl, x, u, v, a if scheme == 2 else None)
    assert _eq(xo, ref["x"]) and _eq(uo, ref["u"]) and _eq(vo, ref["v"])
    if scheme == 2:
        assert _eq(ao, ref["a"])
    assert bb in (1, 4)


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", [1, 2])
def test_device_newmark_matches_oracle(ctx, scheme):
    torch = pytest.importorskip("torch")
    from delfem_b200 import lib
    m, b, rp, ci, params, u, v, a, x = _case(scheme, n=24, seed=3)
    rng = np.random.default_rng(7)
    N = m.nnode
    kd, ko = rng.standard_normal(N * b * b), rng.standard_normal(ci.size * b * b)
    fl = np.zeros(N * b, np.int32)
    fl[np.unique(m.bnd.ravel())[:, None] * b + np.arange(b)] = 1
    force = rng.standard_normal(N * b)
    dev = lambda t: torch.from_numpy(np.ascontiguousarray(t)).cuda()  # noqa: E731
    B = lib.Matrix(ctx, rp, ci, b)
    B.set_values(kd, ko)
    fl_d = dev(fl)
    lib.mat_zero_rows(B, fl_d)
    zd, zo = P.mat_zero_rows(N, b, rp, fl, kd, ko)
    gd, go = B.get_values()
    assert _eq(gd, zd) and _eq(go, zo)
    t, r = torch.zeros(N * b, dtype=torch.float64, device="cuda"), torch.zeros(N * b, dtype=torch.float64,
                                                                               device="cuda")
    av = a if scheme == 2 else None
    nrm = lib.newmark_residual(B, scheme, DT, GAMMA, BETA, dev(force), dev(u), dev(v),
                               dev(a) if scheme == 2 else None, fl_d, t, r)
    r_o, nrm_o = P.newmark_residual(N, b, rp, ci, zd, zo, scheme, DT, GAMMA, BETA, force, u, v, av, fl)
    rg = r.cpu().numpy()
    assert np.allclose(rg, r_o, rtol=1e-12, atol=1e-13 * np.abs(r_o).max())
    assert nrm == pytest.approx(nrm_o, rel=1e-12)
    assert not rg[fl != 0].any()
    xd, ud, vd = dev(x), dev(u), dev(v)
    ad = dev(a) if scheme == 2 else None
    lib.newmark_update(ctx, scheme, DT, GAMMA, BETA, fl_d, xd, ud, vd, ad)
    ctx.sync()
    xo, uo, vo, ao = P.newmark_update(scheme, DT, GAMMA, BETA, fl, x, u, v, av)
    assert _eq(xd.cpu().numpy(), xo) and _eq(ud.cpu().numpy(), uo) and _eq(vd.cpu().numpy(), vo)
    if scheme == 2:
        assert _eq(ad.cpu().numpy(), ao)
