"""The complex matrix text reader (dfm_zmat_read_text, host only) against the
reference's own reader CZMatDia_BlkCrs(file_path)
(src/matvec/zmatdia_blkcrs.cpp:108-173), and on the GPU a PCOCG solve of a
matrix read from a file against the oracle."""
import numpy as np
import pytest

from oracle import refshim as R
from tests import cases


def _helmholtz():
    m, S = cases.helmholtz(8)
    return S


def test_reader_matches_reference(tmp_path):
    if not R.available():
        pytest.skip("reference build (oracle/_ref) not present")
    from delfem_b200 import lib
    S = _helmholtz()
    p = tmp_path / "helmholtz.txt"
    cases.write_zmat_text(str(p), S.rowptr, S.colind, S.diag, S.off)
    got = lib.read_complex_matrix_text(str(p))
    ref = R.zmat_read(str(p))
    assert got[0] == ref[0] == S.N
    for a, b in zip(got[1:], ref[1:]):
        assert np.array_equal(a, b)
    # and the values are the system's, bit for bit
    assert np.array_equal(got[3], S.diag) and np.array_equal(got[4], S.off)
    assert np.array_equal(got[1], S.rowptr) and np.array_equal(got[2], S.colind)


def test_reader_matches_reference_fixture():
    """tests/golden/zmat_helmholtz_r4.txt as the reference read it
    (tests/golden/make_golden.py): rows 2 and 5 lack a diagonal entry."""
    import os
    from delfem_b200 import lib
    g = os.path.join(os.path.dirname(__file__), "golden")
    ref = np.load(os.path.join(g, "zmatref_helmholtz_r4.npz"))
    N, rp, ci, d, o = lib.read_complex_matrix_text(os.path.join(g, "zmat_helmholtz_r4.txt"))
    assert N == int(ref["N"])
    for a, k in zip((rp, ci, d, o), ("rowptr", "colind", "diag", "off")):
        assert np.array_equal(a, ref[k]), k


def test_reader_edge_cases(tmp_path):
    from delfem_b200 import lib
    S = _helmholtz()
    # shuffled columns inside rows: read back sorted
    p = tmp_path / "shuffled.txt"
    cases.write_zmat_text(str(p), S.rowptr, S.colind, S.diag, S.off, shuffle_rows=np.random.default_rng(1))
    N, rp, ci, d, o = lib.read_complex_matrix_text(str(p))
    assert np.array_equal(rp, S.rowptr) and np.array_equal(ci, S.colind)
    assert np.array_equal(d, S.diag) and np.array_equal(o, S.off)
    # rows without a diagonal entry: zero diagonal (the reference zeroes it too)
    p = tmp_path / "nodiag.txt"
    cases.write_zmat_text(str(p), S.rowptr, S.colind, S.diag, S.off, skip_diag=(3, 7))
    N, rp, ci, d, o = lib.read_complex_matrix_text(str(p))
    assert d[6] == d[7] == d[14] == d[15] == 0.0 and np.array_equal(o, S.off)
    if R.available():
        ref = R.zmat_read(str(p))
        for a, b in zip((rp, ci, d, o), ref[1:]):
            assert np.array_equal(a, b)
    # empty rows at the start, in the middle and at the end
    p = tmp_path / "empty.txt"
    p.write_text("6 4\n1 1 2.0 0.5\n1 3 -1.0 0.0\n3 1 -1.0 0.0\n3 3 2.5 -0.25\n")
    N, rp, ci, d, o = lib.read_complex_matrix_text(str(p))
    assert N == 6 and list(rp) == [0, 0, 1, 1, 2, 2, 2] and list(ci) == [3, 1]
    assert list(d) == [0, 0, 2.0, 0.5, 0, 0, 2.5, -0.25, 0, 0, 0, 0] and list(o) == [-1.0, 0.0, -1.0, 0.0]
    # an empty matrix
    p = tmp_path / "zero.txt"
    p.write_text("0 0\n")
    N, rp, ci, d, o = lib.read_complex_matrix_text(str(p))
    assert N == 0 and list(rp) == [0] and ci.size == 0


@pytest.mark.parametrize("text", [
    "3 2\n0 0 1 0\n",                      # fewer entries than announced
    "3 2\n1 1 1 0\n0 0 1 0\n",             # decreasing row
    "3 1\n0 3 1 0\n",                      # column out of range
    "3 1\n-1 0 1 0\n",                     # negative row
    "3 2\n0 1 1 0\n0 1 2 0\n",             # repeated off-diagonal entry
    "3 1\n0 1 x 0\n",                      # unparsable value
    "-1 0\n",                              # negative size
    "3 999999999999999\n0 0 1 0\n",        # a count the file cannot hold (no allocation sized by it)
])
def test_reader_rejects_malformed(tmp_path, text):
    from delfem_b200 import lib
    p = tmp_path / "bad.txt"
    p.write_text(text)
    with pytest.raises(lib.DfmError) as e:
        lib.read_complex_matrix_text(str(p))
    assert e.value.code == lib.ERR_INVALID


def test_reader_missing_file(tmp_path):
    from delfem_b200 import lib
    with pytest.raises(lib.DfmError) as e:
        lib.read_complex_matrix_text(str(tmp_path / "absent.txt"))
    assert e.value.code == lib.ERR_IO


@pytest.mark.gpu
def test_pcocg_on_matrix_read_from_file(ctx, tmp_path):
    """A matrix read from the reference's text format solves like the
    assembled one: complex ILU(0)-COCG to 1e-8 of the oracle's x."""
    torch = pytest.importorskip("torch")
    from delfem_b200 import lib
    S = _helmholtz()
    p = tmp_path / "helmholtz.txt"
    cases.write_zmat_text(str(p), S.rowptr, S.colind, S.diag, S.off)
    N, rp, ci, d, o = lib.read_complex_matrix_text(str(p))
    A = lib.Matrix(ctx, rp, ci, 1, lib.COMPLEX)
    A.set_values(d, o)
    M = lib.ILU(A)
    M.factor()
    ns, fd, fo = S.ilu0()
    ref = S.solve(fd, fo, method="pcocg", tol=1e-10, maxit=3000)
    r = torch.from_numpy(S.rhs.copy()).cuda()
    x = torch.zeros_like(r)
    rc, it, conv = lib.solve_pcocg(A, M, r, x, tol=1e-10, maxit=3000)
    assert rc == lib.OK
    xr = ref["x"]
    assert np.linalg.norm(x.cpu().numpy() - xr) <= 1e-8 * np.linalg.norm(xr)
