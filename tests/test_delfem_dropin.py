"""A DelFEM program switched to the device library through
include/dfm_b200_delfem.hpp (tests/cpp/delfem_dropin.cpp, built against the
reference's headers and library by `make -C oracle dropin`): the reference's
field world, assembly, Dirichlet elimination and UpdateValueOfField, with
dfm_delfem::CPreconditioner_ILU_GPU, CLinearSystemGPU and Solve_*_GPU in place
of LsSol's classes.  The same program runs the reference's own solvers on the
same problem (a system of two segments - the reference's block ILU over
segments, src/ls/preconditioner.cpp:57-335, against the drop-in's ILU(0) of
the joined matrix - among them); the field after UpdateValueOfField (the
segments' updates for the two-segment system) must agree to 1e-8 relative
at a relative residual of 1e-10, and the iteration counts within the few that
the device's summation order moves them."""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "delfem_dropin")
X_TOL = 1e-8

pytestmark = pytest.mark.skipif(not os.path.exists(DROPIN),
                                reason="oracle/_ref/delfem_dropin not built (needs the reference tree at build time)")


def test_dropin_program_is_linked_against_the_reference():
    """The program exists and names the reference's solver entry points (it is
    a DelFEM program, not a rewrite)."""
    syms = subprocess.run(["nm", "-C", DROPIN], capture_output=True, text=True).stdout
    for name in ("LsSol::Solve_PCG", "LsSol::CPreconditioner_ILU::SetValue",
                 "Fem::Ls::CLinearSystem_Field::UpdateValueOfField"):
        assert name in syms, name


def _run(args):
    r = subprocess.run([DROPIN, *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout)


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


CASES = [("poisson", ["poisson", "32"]), ("poisson_ilu1", ["poisson", "24", "1"]),
         ("solid3d", ["solid3d", "10", "3", "3"]), ("solid3d_ilu1", ["solid3d", "8", "2", "2", "1"]),
         # two segments (LsSol::CLinearSystem::AddLinSysSeg x 2 with couplings both ways): equal block
         # lengths, and different ones (joined one row per DOF)
         ("twoseg_2_2", ["twoseg", "40", "200", "2", "2"]), ("twoseg_2_1", ["twoseg", "40", "200", "2", "1"]),
         ("twoseg_1_3", ["twoseg", "40", "200", "1", "3"]),
         # ILU(k) across the segments: the joined matrix's ILU(k) against the reference's segment-wise one
         ("twoseg_2_2_ilu1", ["twoseg", "40", "200", "2", "2", "1"]),
         ("twoseg_2_1_ilu2", ["twoseg", "40", "200", "2", "1", "2"]),
         # CPreconditioner_ILU::SetOrdering: the rows reversed or shuffled (ILU(0) of the renumbered matrix)
         ("poisson_ord_rev", ["poisson", "24", "0", "rev"]), ("poisson_ord_rand", ["poisson", "32", "0", "rand"]),
         ("solid3d_ord_rand", ["solid3d", "10", "3", "3", "0", "rand"]),
         # CPreconditioner_ILU::SetFillBlk: unlimited fill through listed block rows (AddFracPtn(lev, aBlkFill))
         ("poisson_fill_ilu1", ["poisson", "32", "1", "fill"]), ("solid3d_fill_ilu0", ["solid3d", "10", "3", "3", "0", "fill"]),
         ("twoseg_2_2_fill_ilu1", ["twoseg", "40", "200", "2", "2", "1", "fill"]),
         ("twoseg_2_1_fill_ilu0", ["twoseg", "40", "200", "2", "1", "0", "fill"])]


@pytest.mark.gpu
@pytest.mark.parametrize("name,args", CASES, ids=[c[0] for c in CASES])
def test_dropin_matches_reference(name, args):
    out = _run(args)
    ref_pcg, ref_bicg, ref_cg = out["ref_pcg"], out["ref_bicg"], out["ref_cg"]
    assert ref_pcg["ok"] and ref_bicg["ok"] and ref_cg["ok"]
    assert max(abs(v) for v in ref_pcg["x"]) > 0  # the field was updated
    # the drop-in's fused device solves
    for run, ref, slack in (("gpu_pcg", ref_pcg, 1), ("gpu_bicg", ref_bicg, 2), ("gpu_cg", ref_cg, 3)):
        g = out[run]
        assert g["ok"], run
        assert abs(g["iters"] - ref["iters"]) <= max(slack, ref["iters"] // 50), (run, g["iters"], ref["iters"])
        assert g["conv"] < 1e-10, run
        assert _rel(g["x"], ref["x"]) <= X_TOL, (run, _rel(g["x"], ref["x"]))
    # the reference's own Solve_PCG over the device-backed interface, and the
    # reference's glue class with the device preconditioner
    for run in ("ref_over_gpu", "glue_gpu_prec"):
        g = out[run]
        assert g["ok"] and abs(g["iters"] - ref_pcg["iters"]) <= 1, (run, g["iters"], ref_pcg["iters"])
        assert _rel(g["x"], ref_pcg["x"]) <= X_TOL, run
