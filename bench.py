"""Benchmark of the B200 linear-solve path on the 3D cantilever elasticity
system (200x40x40 hexes x 6 P1 tets, 337,881 nodes, 1,013,643 DOF, 3x3 blocks).

One step = one complete solve as the reference performs it after assembly:
numeric ILU(0) of K (CPreconditioner_ILU::SetValue) followed by ILU(0)-PCG to
relative residual 1e-8 from x = 0 (LsSol::Solve_PCG).  Inputs (K, f) are
generated once (seeded, deterministic mesh; E = 1, nu = 0.3, body force -z,
x = 0 face clamped) and are larger than L2 (K is 354 MB).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  Under torchrun every rank solves its own
replica (the single-system path does not shard: "replicas only"); the value
is the solves/s of all ranks, timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solve time to rel.res 1e-8: mixed/batched vs plain FP64 GPU PCG; SpMV HBM GB/s"
UNIT = "solves/s (c2, rel.res 1e-8)"
TOL = 1e-8
NX, NY, NZ = 200, 40, 40


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------ workload
def build_system():
    from delfem_b200 import meshes
    from oracle import port as P
    from tests import cases
    t0 = time.time()
    m = meshes.box_tet(NX, NY, NZ)
    rp, ci = P.pattern(m.nnode, m.elem)
    S = P.System(rp, ci, 3)
    S.asm_solid3d(m, cases.LAM3, cases.MYU3, 1.0, 0.0, 0.0, -1.0)
    S.apply_bc(P.bc_flags_from_bnd(m.nnode, 3, m.bnd))
    log(f"[bench] c2 system N={S.N} ncrs={S.ncrs} built in {time.time() - t0:.1f}s")
    return m, S


def alg_bytes(N, ncrs, b, sv=8, sx=8):
    bb = b * b
    spmv = (ncrs + N) * bb * sv + 4 * ncrs + 4 * (N + 1) + 2 * N * b * sx
    ilu = (ncrs + N) * bb * sv + 4 * ncrs + 4 * (N + 1) + 4 * N + 4 * N * b * sx
    it = spmv + ilu + 10 * N * b * sx
    return spmv, ilu, it


# ------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([s.strip() for s in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and "Active" in r[5 + k]
                          and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------- reference arm
def reference_runs():
    p = os.path.join(ROOT, "tests", "golden", "reference_runs.json")
    return json.load(open(p)) if os.path.exists(p) else {}


def cpu_reference_sample(S, sample_iters):
    """The reference's own ILU(0) + Solve_PCG (oracle/_ref, built from its
    sources) on a bounded sample: ILU + `sample_iters` PCG iterations, scaled to
    a full solve with the reference's iteration count to 1e-8."""
    from oracle import refshim as R
    rc, x, it, conv, t_ilu, t_solve = R.mat_solve(S.N, S.b, S.rowptr, S.colind, S.diag, S.off, S.rhs,
                                                  R.PCG, TOL, sample_iters)
    t_iter = t_solve / max(sample_iters, 1)
    runs = reference_runs().get("c2", {}).get(f"tol{TOL:g}", {})
    n_full = runs.get("iterations")
    return t_ilu, t_iter, n_full


def run_reference(args, rank):
    if rank != 0:
        return
    _, S = build_system()
    from oracle import refshim as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libdfm_refshim.so was not built"}))
        return
    per_step = []
    n_full = None
    for k in range(args.warmup + args.steps):
        t_ilu, t_iter, n_full = cpu_reference_sample(S, 5)
        if n_full is None:
            n_full = 1
        if k >= args.warmup:
            per_step.append(t_ilu + n_full * t_iter)
    t = statistics.median(per_step)
    v = 1.0 / t
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": "c2 3D elasticity 200x40x40x6 tets, ILU(0)+PCG to 1e-8",
                       "N": S.N, "b": 3, "ncrs": S.ncrs},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                             "sample": f"per step: reference ILU(0) + 5 Solve_PCG iterations on one core, "
                                       f"scaled to the reference's {n_full} iterations to 1e-8"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# -------------------------------------------------------------------- our arm
def run_ours(args, rank, world):
    import torch
    from delfem_b200 import lib
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    _, S = build_system()
    N, b, ncrs = S.N, S.b, S.ncrs
    stream = torch.cuda.Stream(device=dev)
    ctx = lib.Context(dev)
    lib.check(lib.lib().dfm_ctx_set_stream(ctx.h, lib.C.c_void_p(stream.cuda_stream)))
    A = lib.Matrix(ctx, S.rowptr, S.colind, b)
    A.set_values(S.diag, S.off)
    M = lib.ILU(A)
    b_dev = torch.from_numpy(S.rhs).cuda(dev)
    r = torch.empty_like(b_dev)
    x = torch.empty_like(b_dev)
    torch.cuda.synchronize()

    def step():
        M.factor()
        r.copy_(b_dev)
        torch.cuda.synchronize()
        return lib.solve_pcg(A, M, r, x, tol=TOL, maxit=20000)

    for _ in range(args.warmup):
        rc, iters, conv = step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(dev) as clk:
        torch.cuda.synchronize()
        for k in range(args.steps):
            ev[k][0].record(stream)
            rc, iters, conv = step()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    times = [a.elapsed_time(b_) / 1e3 for a, b_ in ev]
    t_step = sum(times) / len(times)
    if world > 1:
        tt = torch.tensor([t_step], device=f"cuda:{dev}")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        torch.distributed.barrier()
        t_step = float(tt.item())
    x_np = x.cpu().numpy()

    # ---- kernel breakdown (CUDA events on the library stream) ----
    def timed(fn, reps):
        out = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1) / 1e3)
        return statistics.median(out)

    y = torch.empty_like(b_dev)
    t_spmv = timed(lambda: A.spmv(1.0, x, 0.0, y), 20)
    t_apply = timed(lambda: M.apply(r, y), 10)
    t_factor = timed(lambda: M.factor(), 3)
    B_spmv, B_ilu, B_it = alg_bytes(N, ncrs, b)
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if peaks else "fallback"
    n_it = iters + 1
    t_iter = (t_step - t_factor) / n_it
    share_sweep = t_apply * n_it / t_step
    share_spmv = t_spmv * n_it / t_step
    kernels = {
        "spmv_bcrs_b3": {"ms": t_spmv * 1e3, "alg_bytes": B_spmv, "gbs": B_spmv / t_spmv / 1e9,
                         "frac": B_spmv / t_spmv / 1e9 / hbm, "share_of_step": share_spmv},
        "ilu0_fwd_bwd": {"ms": t_apply * 1e3, "alg_bytes": B_ilu, "gbs": B_ilu / t_apply / 1e9,
                         "frac": B_ilu / t_apply / 1e9 / hbm, "share_of_step": share_sweep},
        "ilu0_factor": {"ms": t_factor * 1e3},
        "pcg_iteration": {"ms": t_iter * 1e3, "alg_bytes": B_it, "gbs": B_it / t_iter / 1e9},
    }
    dom = "ilu0_fwd_bwd" if share_sweep >= share_spmv else "spmv_bcrs_b3"
    dk = kernels[dom]
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp)).get(dom)

    # ---- end-to-end through the C ABI with host buffers ----
    diag_h = torch.from_numpy(S.diag).pin_memory()
    off_h = torch.from_numpy(S.off).pin_memory()
    b_h = torch.from_numpy(S.rhs).pin_memory()
    x_h = torch.empty_like(b_h).pin_memory()
    L = lib.lib()
    it_c, conv_c = lib.C.c_uint(), lib.C.c_double()

    def e2e_step():
        lib.check(L.dfm_mat_set_values(A.h, lib._ptr(diag_h), lib._ptr(off_h), lib.HOST))
        M.factor()
        lib.check(L.dfm_solve_pcg_host(A.h, M.h, lib._ptr(b_h), lib._ptr(x_h), TOL, 20000, lib.C.byref(it_c),
                                       lib.C.byref(conv_c)), allow=(lib.OK,))

    e2e_step()
    t_e2e = timed(e2e_step, max(2, min(args.steps, 5)))
    h2d = (S.diag.nbytes + S.off.nbytes + S.rhs.nbytes)
    d2h = S.rhs.nbytes

    # ---- parity spot check against the oracle's residual (no oracle solve) ----
    rr = np.linalg.norm(S.rhs - S.spmv(1.0, x_np, 0.0, np.zeros_like(x_np))) / np.linalg.norm(S.rhs)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            t_ilu, t_iter_ref, n_full = cpu_reference_sample(S, 30)
            n_full = n_full or n_it
            v = 1.0 / (t_ilu + n_full * t_iter_ref)
            cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"reference ILU(0) ({t_ilu:.2f}s) + 30 Solve_PCG iterations "
                             f"({t_iter_ref * 1e3:.1f} ms/it) on one host core, scaled to {n_full} iterations",
                   "t_ilu_s": t_ilu, "t_iter_s": t_iter_ref, "iterations": n_full}
        except Exception as e:  # the reference build is optional on a box
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"unavailable: {e}"}

    launches = 1 + 4 + 16 * ((n_it + 15) // 16) * 5
    if rank == 0:
        line = {
            "metric": METRIC, "value": world / t_step, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "c2 3D elasticity cantilever 200x40x40 hexes x 6 P1 tets, ILU(0) + PCG to "
                                   "rel.res 1e-8 (plain FP64)", "N": N, "b": b, "ncrs": ncrs,
                       "dof": N * b, "l2": "inputs larger than L2 (K = %.0f MB)" % (S.off.nbytes / 1e6),
                       "parallelism": f"replicas x{world}"},
            "iterations": n_it, "conv": conv, "true_rel_residual": rr,
            "solve_time_s": t_step,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": dk["gbs"], "peak": hbm, "unit": "GB/s",
                         "frac": dk["frac"], "traffic": traffic, "peak_source": peak_src},
            "spmv_roofline": {"achieved": kernels["spmv_bcrs_b3"]["gbs"], "peak": hbm, "unit": "GB/s",
                              "frac": kernels["spmv_bcrs_b3"]["frac"]},
            "kernels": kernels,
            "e2e": {"value": 1.0 / t_e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": t_e2e * 1e3},
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": clk.summary(),
        }
        print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
