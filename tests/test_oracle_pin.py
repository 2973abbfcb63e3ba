"""Pins the oracle's C restatement to the reference's own code on seeded cases
larger than the fixtures (skipped where the reference build, oracle/_ref/
libdfm_refshim.so, is absent): pattern, assembly, elimination, ILU(0),
preconditioner and solves must be bit-identical."""
import numpy as np
import pytest

from delfem_b200 import meshes
from oracle import port as P
from oracle import refshim as R
from tests import cases

pytestmark = pytest.mark.skipif(not R.available(), reason="reference build (oracle/_ref) not present")


def _eq(a, b):
    return np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


CASES = [
    ("poisson", R.POISSON2D, lambda: meshes.unit_square_tri(20), [1.3, 0.7], True, False, "pcg"),
    ("solid2d", R.SOLID2D, lambda: meshes.unit_square_tri(12, bnd="left"),
     [cases.LAM2_PS, cases.MYU2, 0.5, 0.0, -1.0], True, True, "pcg"),
    ("solid3d", R.SOLID3D, lambda: meshes.box_tet(8, 3, 3), [cases.LAM3, cases.MYU3, 1.0, 0.0, 0.0, -1.0], False,
     False, "pbicgstab"),
    ("helmholtz", R.HELMHOLTZ2D, lambda: meshes.unit_disk_tri(16), [2 * 3.1416 / 6], False, True, "pcocg"),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_oracle_pinned_to_reference(case):
    name, kind, mk, params, with_coef, with_load, method = case
    m = mk()
    rng = np.random.default_rng(11)
    coef = rng.lognormal(0, 0.7, m.elem.shape[0]) if with_coef else None
    load = None
    if with_load:
        load = meshes.gaussian_source_load(m) if kind == R.HELMHOLTZ2D else meshes.right_edge_traction(m, 12)
    ref = R.RefSystem(kind, m)
    rp, ci = ref.pattern()
    ref.assemble(params, coef, load)
    d, o, rhs = ref.system()
    ref.ilu()
    _, fd, fo = ref.ilu_factor()
    rc, x, it, conv, _ = ref.solve({"pcg": R.PCG, "pbicgstab": R.PBICGSTAB, "pcocg": R.PCOCG}[method], 1e-10, 3000)

    prp, pci = P.pattern(m.nnode, m.elem)
    assert np.array_equal(prp, rp) and np.array_equal(pci, ci)
    b = {R.POISSON2D: 1, R.SOLID2D: 2, R.SOLID3D: 3, R.HELMHOLTZ2D: 1}[kind]
    S = P.System(rp, ci, b, cplx=kind == R.HELMHOLTZ2D)
    if kind == R.POISSON2D:
        S.asm_poisson(m, *params, coef)
    elif kind == R.SOLID2D:
        S.asm_solid2d(m, *params, coef)
    elif kind == R.SOLID3D:
        S.asm_solid3d(m, *params)
    else:
        S.asm_helmholtz(m, params[0])
    if load is not None:
        S.rhs += np.asarray(load).ravel()
    if kind != R.HELMHOLTZ2D:
        flags = P.bc_flags_from_bnd(m.nnode, b, m.bnd)
        assert np.array_equal(flags, ref.bcflag())
        S.apply_bc(flags)
    assert _eq(S.diag, d) and _eq(S.off, o) and _eq(S.rhs, rhs)
    ns, pfd, pfo = S.ilu0()
    assert _eq(pfd, fd) and _eq(pfo, fo)
    out = S.solve(pfd, pfo, method=method, tol=1e-10, maxit=3000)
    assert out["iters"] == it and out["conv"] == conv and _eq(out["x"], x)
    assert out["ok"] == (rc == 0)
