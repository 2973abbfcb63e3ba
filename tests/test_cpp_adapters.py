"""The reference-shaped C++ adapters (include/dfm_b200_lsol.hpp): a C++ program
using only them and the C ABI compiles and links against the library on the
CPU; on a GPU it solves 2-D Poisson and matches the oracle."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "delfem_b200", "_lib")


@pytest.fixture(scope="module")
def demo(tmp_path_factory):
    from delfem_b200 import build
    build.build()
    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no C++ compiler")
    out = str(tmp_path_factory.mktemp("cpp") / "lsol_demo")
    cmd = [gxx, "-std=c++17", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "lsol_demo.cpp"), "-L", LIBDIR, "-ldfm_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_adapter_program_compiles_and_links(demo):
    assert os.path.exists(demo)


@pytest.mark.gpu
def test_adapter_reads_complex_matrix_text(demo, tmp_path):
    """CMatDia_BlkCrs::FromTextFile (CZMatDia_BlkCrs(file_path)) + PCOCG from a
    C++ program, against the oracle's COCG on the same system.  The disk has 40
    rings (N = 4,921; the oracle's COCG converges in 368 iterations), where
    the iteration count is set by the spectrum, not by rounding."""
    from tests import cases
    m, S = cases.helmholtz(40)
    mp, bp = tmp_path / "z.txt", tmp_path / "b.txt"
    cases.write_zmat_text(str(mp), S.rowptr, S.colind, S.diag, S.off)
    bp.write_text("\n".join(repr(float(v)) for v in S.rhs) + "\n")
    r = subprocess.run([demo, "8", str(mp), str(bp)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout)
    ns, fd, fo = S.ilu0()
    ref = S.solve(fd, fo, method="pcocg", tol=1e-10, maxit=3000)
    assert ref["ok"] and ref["iters"] < 1000
    x = np.array(out["x_file"])
    assert out["pcocg_ok"] and np.linalg.norm(x - ref["x"]) <= 1e-8 * np.linalg.norm(ref["x"])
    assert abs(out["pcocg_iters"] - ref["iters"]) <= max(3, ref["iters"] // 20), (out["pcocg_iters"], ref["iters"])


@pytest.mark.gpu
def test_adapter_program_matches_oracle(demo):
    from delfem_b200 import meshes
    from oracle import port as P
    r = subprocess.run([demo, "16"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout)
    m = meshes.unit_square_tri(16)
    S = P.System(*P.pattern(m.nnode, m.elem), 1)
    S.asm_poisson(m, 1.0, 1.0)
    S.apply_bc(P.bc_flags_from_bnd(m.nnode, 1, m.bnd))
    ns, fd, fo = S.ilu0()
    ref = S.solve(fd, fo, method="pcg", tol=1e-10, maxit=1000)
    refb = S.solve(fd, fo, method="pbicgstab", tol=1e-10, maxit=1000)
    x = np.array(out["x"])
    assert out["pcg_ok"] and abs(out["pcg_iters"] - ref["iters"]) <= 1
    assert np.linalg.norm(x - ref["x"]) <= 1e-8 * np.linalg.norm(ref["x"])
    assert out["bicg_ok"] and abs(out["bicg_iters"] - refb["iters"]) <= 2
    ns1, fpat, fd1, fo1 = S.iluk(1)  # SetFillInLevel(1)
    ref1 = S.solve_fill(fpat, fd1, fo1, tol=1e-10, maxit=1000)
    x1 = np.array(out["x_ilu1"])
    assert out["ilu1_ok"] and abs(out["ilu1_iters"] - ref1["iters"]) <= 1 and ref1["iters"] < ref["iters"]
    assert np.linalg.norm(x1 - ref1["x"]) <= 1e-8 * np.linalg.norm(ref1["x"])
    n = S.N  # SetFillBlk: every 7th block row of the middle third
    ns2, fpat2, fd2, fo2 = S.iluk(1, np.arange(n // 3, 2 * n // 3, 7))
    ref2 = S.solve_fill(fpat2, fd2, fo2, tol=1e-10, maxit=1000)
    x2 = np.array(out["x_fillblk"])
    assert out["fillblk_ok"] and abs(out["fillblk_iters"] - ref2["iters"]) <= 1
    assert np.linalg.norm(x2 - ref2["x"]) <= 1e-8 * np.linalg.norm(ref2["x"])
