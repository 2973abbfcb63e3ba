"""Solutions of the reference's own solvers at the benchmark sizes, kept as
small fixtures: the reference (oracle/_ref/libdfm_refshim.so, built from the
DelFEM sources) assembles each system with its own element routines and
solves it with its own preconditioner and Krylov driver; the fixture holds the
iteration count, the convergence ratio, the 2-norm of x and x at a fixed
stride of entries (the full vectors are megabytes).

    c2       3-D cantilever 200x40x40 hexes x 6 tets (1,013,643 DOF), ILU(0) +
             LsSol::Solve_PCG to rel.res 1e-10 (about three minutes on one core)
    c2half   the same at 100x20x20 (133,623 DOF), to 1e-10
    c5       Helmholtz k = 20 on the unit disk (258 rings, band numbering,
             ~200k nodes), CZPreconditioner_ILU(0) + Fem::Ls::Solve_PCOCG to
             rel.res 1e-8 in complex128

    python tests/golden/make_reference_solutions.py [c2 c2half c5]

Output: tests/golden/reference_solutions.npz (arrays prefixed by the case name).
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from delfem_b200 import meshes  # noqa: E402
from oracle import refshim as R  # noqa: E402
from tests import cases  # noqa: E402

OUT = os.path.join(HERE, "reference_solutions.npz")
STRIDE = {"c2": 61, "c2half": 13, "c5": 61}


def run(name):
    if name in ("c2", "c2half"):
        nx, ny, nz = (200, 40, 40) if name == "c2" else (100, 20, 20)
        m = meshes.box_tet(nx, ny, nz)
        s = R.RefSystem(R.SOLID3D, m)
        s.assemble([cases.LAM3, cases.MYU3, 1.0, 0.0, 0.0, -1.0])
        method, tol = R.PCG, 1e-10
    elif name == "c5":
        m = meshes.unit_disk_tri(258, numbering="bands")
        s = R.RefSystem(R.HELMHOLTZ2D, m)
        s.assemble([cases.WAVE_LENGTH], None, meshes.gaussian_source_load(m))
        method, tol = R.PCOCG, 1e-8
    else:
        raise SystemExit(name)
    s.ilu()
    t0 = time.time()
    rc, x, it, conv, t = s.solve(method, tol, 20000)
    x = np.asarray(x, np.float64)
    if name == "c5":  # complex entries: sample whole (re, im) pairs
        idx = np.arange(0, x.size // 2, STRIDE[name], dtype=np.int64)
        xs = x.reshape(-1, 2)[idx]
    else:
        idx = np.arange(0, x.size, STRIDE[name], dtype=np.int64)
        xs = x[idx]
    print(f"{name}: N={s.N} rc={rc} iterations={it} conv={conv:.3e} |x|={np.linalg.norm(x):.6e} "
          f"solve {t:.1f}s (wall {time.time() - t0:.1f}s)", flush=True)
    return {f"{name}_iters": np.array(it), f"{name}_conv": np.array(conv), f"{name}_ok": np.array(rc == 0),
            f"{name}_xnorm": np.array(np.linalg.norm(x)), f"{name}_idx": idx, f"{name}_x": xs,
            f"{name}_N": np.array(s.N), f"{name}_tol": np.array(tol)}


if __name__ == "__main__":
    if not R.available():
        raise SystemExit("oracle/_ref/libdfm_refshim.so is missing: build it with `make -C oracle ref`")
    names = sys.argv[1:] or ["c2half", "c5", "c2"]
    data = dict(np.load(OUT)) if os.path.exists(OUT) else {}
    for n in names:
        data.update(run(n))
        np.savez_compressed(OUT, **data)
