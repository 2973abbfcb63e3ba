"""Runs the reference's own solver (oracle/_ref/libdfm_refshim.so, built from
the DelFEM sources) to completion on the benchmark configurations and records
iteration counts, final relative residuals and single-core times in
tests/golden/reference_runs.json.

The bench's CPU baseline times a bounded sample of the reference (ILU + a few
PCG iterations) and scales it to a full solve with these iteration counts.

    python tests/golden/make_reference_runs.py [c1|c2|c4 ...]
"""
from __future__ import annotations

import json
import os
import platform
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from delfem_b200 import meshes  # noqa: E402
from oracle import refshim as R  # noqa: E402
from tests import cases  # noqa: E402

OUT = os.path.join(HERE, "reference_runs.json")


def run(name):
    if name == "c1":
        m = meshes.unit_square_tri(256)
        s = R.RefSystem(R.POISSON2D, m)
        _, t_asm = s.assemble([1.0, 1.0])
    elif name == "c2":
        m = meshes.box_tet(200, 40, 40)
        s = R.RefSystem(R.SOLID3D, m)
        _, t_asm = s.assemble([cases.LAM3, cases.MYU3, 1.0, 0.0, 0.0, -1.0])
    else:
        raise SystemExit(name)
    rc, t_ilu = s.ilu()
    out = {"N": s.N, "b": s.b, "ncrs": s.ncrs, "t_assemble_s": t_asm, "t_ilu_s": t_ilu}
    for tol in (1e-8, 1e-10):
        rc, x, it, conv, t = s.solve(R.PCG, tol, 20000)
        out[f"tol{tol:g}"] = {"ok": rc == 0, "iters_0based": it, "iterations": it + 1, "conv": conv,
                              "t_solve_s": t, "t_per_iter_s": t / (it + 1)}
    out["host"] = platform.processor() or platform.machine()
    out["cores_used"] = 1
    return out


if __name__ == "__main__":
    names = sys.argv[1:] or ["c1", "c2"]
    data = json.load(open(OUT)) if os.path.exists(OUT) else {}
    for n in names:
        t0 = time.time()
        data[n] = run(n)
        data[n]["wall_s"] = time.time() - t0
        print(n, json.dumps(data[n]))
        json.dump(data, open(OUT, "w"), indent=1, sort_keys=True)
