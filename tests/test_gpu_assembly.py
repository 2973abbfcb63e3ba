"""Device element assembly and Dirichlet elimination against the oracle's
element loops (oracle/dfm_oracle.c, pinned to the reference): the matrix
values and the residual must be bit-identical, for every element kind, with
and without per-element coefficients, a current field u and nodal loads."""
import numpy as np
import pytest

from delfem_b200 import meshes
from oracle import port as P
from tests import cases

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _dev(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype).cuda()


def _same(got, ref, what):
    assert got.shape == ref.shape, what
    bad = np.flatnonzero(got != ref)
    assert bad.size == 0, f"{what}: {bad.size} entries differ, first {bad[:5]} {got[bad[:3]]} vs {ref[bad[:3]]}"


def _gpu_system(ctx, m, b, cplx=False):
    from delfem_b200 import lib
    rp, ci = P.pattern(m.nnode, m.elem)
    A = lib.Matrix(ctx, rp, ci, b, lib.COMPLEX if cplx else lib.REAL)
    G = lib.Mesh(ctx, m.coord, m.elem, m.bnd if cplx else None)
    S = P.System(rp, ci, b, cplx=cplx)
    return A, G, S


@pytest.mark.parametrize("n", [1, 7, 24])
@pytest.mark.parametrize("with_coef", [False, True])
@pytest.mark.parametrize("with_u", [False, True])
def test_poisson(ctx, n, with_coef, with_u):
    from delfem_b200 import lib
    m = meshes.unit_square_tri(n)
    A, G, S = _gpu_system(ctx, m, 1)
    rng = np.random.default_rng(n)
    coef = rng.lognormal(0, 0.5, m.elem.shape[0]) if with_coef else None
    u = rng.standard_normal(m.nnode) if with_u else None
    load = rng.standard_normal(m.nnode)
    S.asm_poisson(m, 1.3, 0.7, coef, u)
    S.rhs += load
    rhs = torch.full((m.nnode,), float("nan"), dtype=torch.float64, device="cuda")
    A.set_values(np.full(S.diag.size, np.nan), np.full(max(S.off.size, 1), np.nan)[: S.off.size])
    G.assemble_poisson(A, 1.3, 0.7, rhs, None if coef is None else _dev(coef), None if u is None else _dev(u),
                       _dev(load))
    d, o = A.get_values()
    _same(d, S.diag, "diag")
    _same(o, S.off, "off")
    _same(rhs.cpu().numpy(), S.rhs, "rhs")
    flags = P.bc_flags_from_bnd(m.nnode, 1, m.bnd)
    S.apply_bc(flags)
    lib.apply_dirichlet(A, _dev(flags, torch.int32), rhs)
    d, o = A.get_values()
    _same(d, S.diag, "diag after bc")
    _same(o, S.off, "off after bc")
    _same(rhs.cpu().numpy(), S.rhs, "rhs after bc")


@pytest.mark.parametrize("n", [3, 16])
def test_solid2d(ctx, n):
    from delfem_b200 import lib
    m = meshes.unit_square_tri(n, bnd="left")
    A, G, S = _gpu_system(ctx, m, 2)
    rng = np.random.default_rng(5)
    theta = rng.lognormal(0, 0.5, m.elem.shape[0])
    u = rng.standard_normal(2 * m.nnode)
    load = meshes.right_edge_traction(m, n).ravel()
    S.asm_solid2d(m, cases.LAM2_PS, cases.MYU2, 0.8, 0.1, -1.0, theta, u)
    S.rhs += load
    rhs = torch.empty(2 * m.nnode, dtype=torch.float64, device="cuda")
    G.assemble_solid2d(A, cases.LAM2_PS, cases.MYU2, 0.8, 0.1, -1.0, rhs, _dev(theta), _dev(u), _dev(load))
    d, o = A.get_values()
    _same(d, S.diag, "diag")
    _same(o, S.off, "off")
    _same(rhs.cpu().numpy(), S.rhs, "rhs")
    flags = P.bc_flags_from_bnd(m.nnode, 2, m.bnd)
    S.apply_bc(flags)
    lib.apply_dirichlet(A, _dev(flags, torch.int32), rhs)
    d, o = A.get_values()
    _same(d, S.diag, "diag after bc")
    _same(o, S.off, "off after bc")
    _same(rhs.cpu().numpy(), S.rhs, "rhs after bc")


@pytest.mark.parametrize("dims", [(1, 1, 1), (6, 3, 2), (20, 4, 4)])
def test_solid3d(ctx, dims):
    from delfem_b200 import lib
    m = meshes.box_tet(*dims)
    A, G, S = _gpu_system(ctx, m, 3)
    u = np.random.default_rng(3).standard_normal(3 * m.nnode)
    S.asm_solid3d(m, cases.LAM3, cases.MYU3, 1.0, 0.0, 0.0, -1.0, u)
    rhs = torch.empty(3 * m.nnode, dtype=torch.float64, device="cuda")
    G.assemble_solid3d(A, cases.LAM3, cases.MYU3, 1.0, 0.0, 0.0, -1.0, rhs, _dev(u))
    d, o = A.get_values()
    _same(d, S.diag, "diag")
    _same(o, S.off, "off")
    _same(rhs.cpu().numpy(), S.rhs, "rhs")
    flags = P.bc_flags_from_bnd(m.nnode, 3, m.bnd)
    S.apply_bc(flags)
    lib.apply_dirichlet(A, _dev(flags, torch.int32), rhs)
    d, o = A.get_values()
    _same(d, S.diag, "diag after bc")
    _same(o, S.off, "off after bc")
    _same(rhs.cpu().numpy(), S.rhs, "rhs after bc")


@pytest.mark.parametrize("nring", [1, 6, 20])
@pytest.mark.parametrize("with_u", [False, True])
def test_helmholtz(ctx, nring, with_u):
    m = meshes.unit_disk_tri(nring)
    A, G, S = _gpu_system(ctx, m, 1, cplx=True)
    rng = np.random.default_rng(nring)
    u = rng.standard_normal(2 * m.nnode) if with_u else None
    load = meshes.gaussian_source_load(m).ravel()
    S.asm_helmholtz(m, cases.WAVE_LENGTH, u)
    S.rhs += load
    rhs = torch.empty(2 * m.nnode, dtype=torch.float64, device="cuda")
    G.assemble_helmholtz(A, cases.WAVE_LENGTH, rhs, None if u is None else _dev(u), _dev(load))
    d, o = A.get_values()
    _same(d, S.diag, "diag")
    _same(o, S.off, "off")
    _same(rhs.cpu().numpy(), S.rhs, "rhs")


def test_reassembly_overwrites(ctx):
    """Assembling twice gives the same values (InitializeMarge zeroes first)."""
    m = meshes.unit_square_tri(9)
    A, G, S = _gpu_system(ctx, m, 1)
    rhs = torch.empty(m.nnode, dtype=torch.float64, device="cuda")
    G.assemble_poisson(A, 1.0, 1.0, rhs)
    d1, o1 = A.get_values()
    r1 = rhs.cpu().numpy().copy()
    G.assemble_poisson(A, 1.0, 1.0, rhs)
    d2, o2 = A.get_values()
    _same(d2, d1, "diag")
    _same(o2, o1, "off")
    _same(rhs.cpu().numpy(), r1, "rhs")


def test_argument_errors(ctx):
    from delfem_b200 import lib
    m = meshes.unit_square_tri(4)
    A, G, S = _gpu_system(ctx, m, 1)
    rhs = torch.empty(m.nnode, dtype=torch.float64, device="cuda")
    with pytest.raises(lib.DfmError):  # b = 1 matrix for a b = 2 kind
        G.assemble_solid2d(A, 1.0, 1.0, 0.0, 0.0, 0.0, rhs)
    with pytest.raises(lib.DfmError):  # node index out of range
        lib.Mesh(ctx, m.coord, np.array([[0, 1, m.nnode]], np.int32))


@pytest.mark.parametrize("mk", [lambda: meshes.unit_square_tri(13), lambda: meshes.box_tet(5, 3, 2),
                                lambda: meshes.unit_disk_tri(9), lambda: meshes.unit_square_tri(1)],
                         ids=["square", "box", "disk", "two_tris"])
def test_mesh_pattern_is_the_references(ctx, mk):
    """The library's own pattern builder against the oracle's (pinned to AddPattern)."""
    from delfem_b200 import lib
    m = mk()
    G = lib.Mesh(ctx, m.coord, m.elem)
    rp, ci = G.pattern()
    prp, pci = P.pattern(m.nnode, m.elem)
    assert np.array_equal(rp, prp) and np.array_equal(ci, pci)
