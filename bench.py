"""Benchmark of the B200 linear-solve path.

Headline workload (the `value`): the 3D cantilever elasticity system, a
200x40x40 hex grid split into 6 P1 tetrahedra each (337,881 nodes, 1,013,643
DOF, 3x3 blocks, E = 1, nu = 0.3, body force -z, x = 0 face clamped).  One step
= one complete solve as the reference performs it after assembly: numeric
ILU(0) of K (CPreconditioner_ILU::SetValue) and ILU(0)-PCG from x = 0 to
relative residual 1e-8 (LsSol::Solve_PCG), plain FP64.  The system is
assembled on the device by the library itself (mesh -> pattern -> element
assembly -> Dirichlet elimination) before timing; K (354 MB of values) is
larger than L2.

Beside it, in the same JSON line:
  mixed    the same c2 solve by dfm_solve_pcg_mixed (FP32 values in SpMV and
           ILU sweeps, FP64 residual replacement) with its error against the
           FP64 solve and its speed-up
  batched  512 uneven 2-D diffusion instances (grid sides log-uniform in
           [32, 512], per-element kappa ~ lognormal(0, 1)) in one batched solve
           against a loop of plain single-instance solves (timed on a
           size-stratified sample of the instances and scaled)
  ilu1     the same c2 solve with ILU(1) (CPreconditioner_ILU::SetFillInLevel(1))
  spmv     SpMV HBM throughput against the measured peak

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--skip-batched] [--skip-mixed] [--skip-iluk] [--no-cpu-baseline]
    python bench.py --profile-run      # short c2 workload for ncu captures


Prints one JSON line (rank 0).  Under torchrun every rank solves its own
replica (a single system does not shard: "replicas only"); the value is the
solves/s of all ranks over the max-over-ranks time.
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
NU = 0.3
LAM3 = NU / ((1 + NU) * (1 - 2 * NU))
MYU3 = 1.0 / (2 * (1 + NU))
C3_COUNT, C3_LO, C3_HI, C3_SEED = 512, 32, 512, 3
C5_MAXIT = 5000  # the oracle's COCG needs 1794 iterations on this system


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def alg_bytes(N, ncrs, b, sv=8, sx=8):
    """Algorithmic bytes of one SpMV, one ILU fwd+bwd application and one PCG
    iteration (values, indices, vectors read/written once)."""
    bb = b * b
    spmv = (ncrs + N) * bb * sv + 4 * ncrs + 4 * (N + 1) + 2 * N * b * sx
    ilu = (ncrs + N) * bb * sv + 4 * ncrs + 4 * (N + 1) + 4 * N + 4 * N * b * sx
    it = spmv + ilu + 10 * N * b * sx
    return spmv, ilu, it


# ------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

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
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 5 + k and "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------ c2 on the GPU
def c2_mesh():
    from delfem_b200 import meshes
    return meshes.box_tet(NX, NY, NZ)


def build_c2(ctx, torch, dev):
    """Pattern, assembly and Dirichlet elimination through the library."""
    from delfem_b200 import lib
    t0 = time.time()
    m = c2_mesh()
    G = lib.Mesh(ctx, m.coord, m.elem)
    rp, ci = G.pattern()
    A = lib.Matrix(ctx, rp, ci, 3)
    rhs = torch.empty(3 * m.nnode, dtype=torch.float64, device=f"cuda:{dev}")
    flags = np.zeros((m.nnode, 3), np.int32)
    flags[np.unique(m.bnd.ravel())] = 1
    flags_d = torch.from_numpy(flags.ravel()).cuda(dev)
    torch.cuda.synchronize()
    t1 = time.time()
    G.assemble_solid3d(A, LAM3, MYU3, 1.0, 0.0, 0.0, -1.0, rhs)
    lib.apply_dirichlet(A, flags_d, rhs)
    torch.cuda.synchronize()
    t_asm = time.time() - t1
    log(f"[bench] c2 N={A.N} ncrs={A.ncrs} set up in {time.time() - t0:.1f}s (device assembly {t_asm * 1e3:.1f} ms)")
    return m, G, A, rhs, t_asm


# ------------------------------------------------------------- reference arm
def reference_runs():
    p = os.path.join(ROOT, "tests", "golden", "reference_runs.json")
    return json.load(open(p)) if os.path.exists(p) else {}


def reference_solution(name):
    """The reference's own solution of a benchmark system at a stride of
    entries, with its norm and iteration count (tests/golden/
    reference_solutions.npz, made by tests/golden/make_reference_solutions.py)."""
    p = os.path.join(ROOT, "tests", "golden", "reference_solutions.npz")
    if not os.path.exists(p):
        return None
    g = np.load(p)
    return {k[len(name) + 1:]: g[k] for k in g.files if k.startswith(name + "_")} or None


def cpu_reference_sample(N, b, rowptr, colind, diag, off, rhs, sample_iters):
    """The reference's own ILU(0) + Solve_PCG (oracle/_ref, built from its
    sources) on a bounded sample: the ILU(0) and `sample_iters` PCG iterations
    timed on one host core."""
    from oracle import refshim as R
    rc, x, it, conv, t_ilu, t_solve = R.mat_solve(N, b, rowptr, colind, diag, off, rhs, R.PCG, TOL, sample_iters)
    return t_ilu, t_solve / max(sample_iters, 1)


C2_CONFIG = {"workload": "c2 3D elasticity cantilever 200x40x40 hexes x 6 P1 tets, ILU(0) + PCG to "
                         "rel.res 1e-8 (plain FP64)", "N": 337881, "b": 3, "ncrs": 4586160, "dof": 1013643,
             "l2": "inputs larger than L2 (K = 330 MB)"}


def run_reference(args, rank):
    """The reference's stock CPU path on c2 (oracle/_ref, built from the
    DelFEM sources): its own pattern, element assembly, ILU(0)
    (CPreconditioner_ILU::SetValue) and LsSol::Solve_PCG, single-threaded.
    One complete solve to 1e-8 is timed in this run and gives the value; the
    K timed steps are bounded samples (the ILU(0) and 5 PCG iterations) whose
    scaled time is reported beside it as a cross-check."""
    if rank != 0:
        return
    from oracle import refshim as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libdfm_refshim.so was not built"}))
        return
    m = c2_mesh()
    s = R.RefSystem(R.SOLID3D, m)
    _, t_asm = s.assemble([LAM3, MYU3, 1.0, 0.0, 0.0, -1.0])
    d, o, rhs = s.system()
    rp, ci = s.pattern()
    per_step, samples = [], []
    for k in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        t_ilu, t_iter = cpu_reference_sample(s.N, s.b, rp, ci, d, o, rhs, 5)
        if k >= args.warmup:
            per_step.append(time.perf_counter() - t0)
            samples.append((t_ilu, t_iter))
    # one complete solve: the field-level ILU(0) and Solve_PCG to 1e-8
    rc_i, t_ilu_full = s.ilu()
    rc, x, it, conv, t_pcg = s.solve(R.PCG, TOL, 20000)
    t_full = t_ilu_full + t_pcg
    n_full = it + 1
    t_ilu_med = statistics.median(a for a, _ in samples)
    t_iter_med = statistics.median(b_ for _, b_ in samples)
    v = 1.0 / t_full
    cfg = dict(C2_CONFIG, parallelism=f"replicas x{args.gpus}")  # the same dict as our arm's
    print(json.dumps({
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.median(per_step) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": cfg,
        "value_basis": f"one complete reference solve timed in this run: ILU(0) {t_ilu_full:.2f}s + Solve_PCG "
                       f"{t_pcg:.1f}s ({n_full} iterations to {TOL:g}); ms_per_step is the median bounded "
                       f"sample (ILU(0) + 5 iterations)",
        "full_solve": {"ilu_s": t_ilu_full, "pcg_s": t_pcg, "iterations": n_full, "conv": conv, "ok": rc == 0,
                       "s_per_iteration": t_pcg / n_full},
        "sample_scaled_solve_s": t_ilu_med + n_full * t_iter_med,
        "reference_assembly_s": t_asm,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                         "sample": f"one full solve ({n_full} iterations) on one host core; steps: the "
                                   f"reference's ILU(0) + 5 Solve_PCG iterations each"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


# --------------------------------------------------------------- c3 batched
def build_c3(ctx, torch, dev):
    from delfem_b200 import lib, meshes
    t0 = time.time()
    sizes = meshes.batch_sizes(C3_COUNT, C3_LO, C3_HI, C3_SEED)
    ms = [meshes.unit_square_tri(int(n)) for n in sizes]
    big, noff, eoff = meshes.concat(ms)
    kappa = np.random.default_rng(C3_SEED + 1).lognormal(0.0, 1.0, big.elem.shape[0])
    G = lib.Mesh(ctx, big.coord, big.elem)
    rp, ci = G.pattern()
    A = lib.Matrix(ctx, rp, ci, 1)
    rhs = torch.empty(big.nnode, dtype=torch.float64, device=f"cuda:{dev}")
    flags = np.zeros(big.nnode, np.int32)
    flags[np.unique(big.bnd.ravel())] = 1
    G.assemble_poisson(A, 1.0, 1.0, rhs, coef=torch.from_numpy(kappa).cuda(dev))
    lib.apply_dirichlet(A, torch.from_numpy(flags).cuda(dev), rhs)
    M = lib.ILU(A)
    M.factor()
    B = lib.Batch(M, noff.astype(np.uint32))
    torch.cuda.synchronize()
    log(f"[bench] c3 {C3_COUNT} instances, {big.nnode} nodes, ncrs={A.ncrs}, set up in {time.time() - t0:.1f}s")
    return sizes, ms, noff, eoff, kappa, A, M, B, rhs


def run_c3(ctx, torch, dev, stream, timed, steps):
    from delfem_b200 import lib
    sizes, ms, noff, eoff, kappa, A, M, B, rhs = build_c3(ctx, torch, dev)
    x = torch.zeros_like(rhs)
    res = {}
    t0 = time.time()
    B.solve(rhs, x, tol=TOL)  # warm-up: autotunes the sweep schedule and the batch tiles
    log(f"[bench] c3 warm-up (tuning) {time.time() - t0:.1f}s: sweep {M.sweep}, schedule {B.schedule}")
    t_batch = timed(lambda: B.solve(rhs, x, tol=TOL), max(2, min(steps, 3)))
    rc, _, it, conv, st = B.solve(rhs, x, tol=TOL)
    log(f"[bench] c3 batched solve {t_batch:.2f}s, max iterations {int(it.max())}")
    t0 = time.time()
    xb = x.cpu().numpy()
    # looped plain solves on a size-stratified sample (every k-th instance by size)
    order = np.argsort(sizes, kind="stable")
    stride = 8
    sample = order[stride // 2::stride]
    t_loop_sample = 0.0
    err = 0.0
    for k in sample:
        a0, a1 = int(noff[k]), int(noff[k + 1])
        m = ms[k]
        Gk = lib.Mesh(ctx, m.coord, m.elem)
        rp, ci = Gk.pattern()
        Ak = lib.Matrix(ctx, rp, ci, 1)
        rk = torch.empty(m.nnode, dtype=torch.float64, device=f"cuda:{dev}")
        fl = np.zeros(m.nnode, np.int32)
        fl[np.unique(m.bnd.ravel())] = 1
        Gk.assemble_poisson(Ak, 1.0, 1.0, rk, coef=torch.from_numpy(kappa[eoff[k]:eoff[k + 1]]).cuda(dev))
        lib.apply_dirichlet(Ak, torch.from_numpy(fl).cuda(dev), rk)
        Mk = lib.ILU(Ak)
        Mk.factor()
        bk = rk.clone()
        xk = torch.zeros_like(bk)
        rwork = bk.clone()
        lib.solve_pcg(Ak, Mk, rwork, xk, tol=TOL, maxit=20000)  # warm-up (autotune + graph capture)

        def one():
            rwork.copy_(bk)
            lib.solve_pcg(Ak, Mk, rwork, xk, tol=TOL, maxit=20000)

        t_loop_sample += timed(one, 1)
        xs = xk.cpu().numpy()
        err = max(err, float(np.linalg.norm(xs - xb[a0:a1]) / max(np.linalg.norm(xs), 1e-300)))
        for h in (Mk, Ak, Gk):
            h.close()
    t_loop = t_loop_sample * (len(sizes) / len(sample))
    log(f"[bench] c3 looped sample {t_loop_sample:.2f}s ({time.time() - t0:.1f}s with set-up and tuning)")
    res.update({
        "instances": int(len(sizes)), "nodes": int(noff[-1]), "grid_sides": [int(sizes.min()), int(sizes.max())],
        "batched_s": t_batch, "looped_s_estimated": t_loop, "speedup_vs_looped": t_loop / t_batch,
        "looped_sample": f"{len(sample)} instances (every {stride}th by size) timed one by one with dfm_solve_pcg, "
                         f"scaled by {len(sizes) / len(sample):.0f}",
        "max_iterations": int(it.max()), "all_converged": bool((st == lib.OK).all()),
        "max_rel_diff_vs_single_solves": err, "tuning": list(B.tuning), "schedule": list(B.schedule),
        "sweep": M.sweep,
    })
    for h in (B, M, A):
        h.close()
    return res


def run_c3_sharded(torch, dev, stream, steps):
    """c3 over all ranks (bench.py --gpus N > 1): the 512 instances shard by a
    greedy balance of (n+1)^2 (delfem_b200.shard), every rank solves its share
    as one batch, the time of a batched solve is the max over ranks (CUDA events
    on this rank's stream, all-reduce over NCCL); the per-instance results are
    gathered to rank 0.  No data-path collective: weak scaling by instances."""
    from delfem_b200 import lib, meshes, shard
    sizes = meshes.batch_sizes(C3_COUNT, C3_LO, C3_HI, C3_SEED)
    nel = 2 * sizes.astype(np.int64) ** 2
    eoff = np.concatenate([[0], np.cumsum(nel)])
    kappa_all = np.random.default_rng(C3_SEED + 1).lognormal(0.0, 1.0, int(eoff[-1]))  # the 1-GPU c3 stream

    def solve_local(idx):
        ctx = lib.Context(dev)
        ms = [meshes.unit_square_tri(int(sizes[k])) for k in idx]
        big, noff, _ = meshes.concat(ms)
        kappa = np.concatenate([kappa_all[eoff[k]:eoff[k + 1]] for k in idx])
        G = lib.Mesh(ctx, big.coord, big.elem)
        rp, ci = G.pattern()
        A = lib.Matrix(ctx, rp, ci, 1)
        rhs = torch.empty(big.nnode, dtype=torch.float64, device=f"cuda:{dev}")
        fl = np.zeros(big.nnode, np.int32)
        fl[np.unique(big.bnd.ravel())] = 1
        G.assemble_poisson(A, 1.0, 1.0, rhs, coef=torch.from_numpy(kappa).cuda(dev))
        lib.apply_dirichlet(A, torch.from_numpy(fl).cuda(dev), rhs)
        M = lib.ILU(A)
        M.factor()
        B = lib.Batch(M, noff.astype(np.uint32))
        x = torch.zeros_like(rhs)
        B.solve(rhs, x, tol=TOL)  # warm-up: autotuning
        ts = []
        for _ in range(max(2, min(steps, 3))):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            rc, _, it, conv, st = B.solve(rhs, x, tol=TOL)
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1) / 1e3)
        res = [(int(it[j]), int(st[j])) for j in range(len(idx))]
        for h in (B, M, A, G):
            h.close()
        ctx.close()
        return statistics.median(ts), res

    out = shard.timed_sharded([(int(n) + 1) ** 2 for n in sizes], solve_local, device=f"cuda:{dev}")
    if out is None:
        return {}
    its = [r[0] for r in out["results"]]
    return {"instances": int(len(sizes)), "per_rank_instances": out["per_rank_instances"],
            "per_rank_s": out["per_rank_seconds"], "batched_s_max_over_ranks": out["seconds"],
            "instances_per_s": len(sizes) / out["seconds"], "max_iterations": int(max(its)),
            "all_converged": all(r[1] == 0 for r in out["results"]), "scaling": "weak (instances)"}


# ------------------------------------------------------------- profile run
def run_profile():
    """A short workload for profiler captures: every kernel family of the path
    runs a few times inside the NVTX range "steady" (after the autotuners),
    each family in a sub-range of its own: c2 assembly + Dirichlet
    elimination, ILU(0) factor, SpMV, ILU applications (FP64 and the FP32
    copy of the mixed solve), a 32-iteration PCG (Krylov update kernels);
    the c5 Helmholtz system (complex assembly, factor, SpMV, sweeps); a batch
    of 64 c3 instances (batched kernels).  No timing output."""
    import torch
    from delfem_b200 import lib, meshes
    ctx = lib.Context(0)
    m, G, A, b_dev, _ = build_c2(ctx, torch, 0)
    M = lib.ILU(A)
    part, nparts = lib.sweep_partition_patches(m.coord, torch.cuda.get_device_properties(0).multi_processor_count)
    M.set_sweep_partition(part, nparts)  # as the bench's c2 solve
    M.factor()
    x = torch.zeros_like(b_dev)
    y = torch.empty_like(b_dev)
    r = b_dev.clone()
    rc, it, conv = lib.solve_pcg(A, M, r, x, tol=TOL, maxit=32)  # autotunes SpMV lanes and the sweep schedule
    r.copy_(b_dev)
    lib.solve_pcg_mixed(A, M, r, x, tol=TOL, maxit=16)  # FP32 factor copy and its plans
    flags = np.zeros((m.nnode, 3), np.int32)
    flags[np.unique(m.bnd.ravel())] = 1
    flags_d = torch.from_numpy(flags.ravel()).cuda()
    # c5 and a c3 subset, tuned before the range
    mz = meshes.unit_disk_tri(258, numbering="bands")
    GZ = lib.Mesh(ctx, mz.coord, mz.elem, mz.bnd)
    AZ = lib.Matrix(ctx, *GZ.pattern(), 1, lib.COMPLEX)
    bz = torch.empty(2 * mz.nnode, dtype=torch.float64, device="cuda")
    loadz = torch.from_numpy(meshes.gaussian_source_load(mz).ravel()).cuda()
    GZ.assemble_helmholtz(AZ, 2 * 3.1416 / 20, bz, load=loadz)
    MZ = lib.ILU(AZ)
    MZ.factor()
    xz, yz, rz = torch.zeros_like(bz), torch.empty_like(bz), bz.clone()
    lib.solve_pcocg(AZ, MZ, rz, xz, tol=1e-8, maxit=16)
    sizes = meshes.batch_sizes(C3_COUNT, C3_LO, C3_HI, C3_SEED)[:64]
    ms = [meshes.unit_square_tri(int(n)) for n in sizes]
    big, noff, _ = meshes.concat(ms)
    GB = lib.Mesh(ctx, big.coord, big.elem)
    AB = lib.Matrix(ctx, *GB.pattern(), 1)
    bb = torch.empty(big.nnode, dtype=torch.float64, device="cuda")
    flb = np.zeros(big.nnode, np.int32)
    flb[np.unique(big.bnd.ravel())] = 1
    GB.assemble_poisson(AB, 1.0, 1.0, bb)
    lib.apply_dirichlet(AB, torch.from_numpy(flb).cuda(), bb)
    MB = lib.ILU(AB)
    MB.factor()
    B = lib.Batch(MB, noff.astype(np.uint32))
    xb = torch.zeros_like(bb)
    B.solve(bb, xb, tol=TOL)  # autotunes the batch schedule
    torch.cuda.synchronize()
    nv = torch.cuda.nvtx
    nv.range_push("steady")  # profiler filter: the tuned steady state only
    nv.range_push("c2_assembly")
    G.assemble_solid3d(A, LAM3, MYU3, 1.0, 0.0, 0.0, -1.0, b_dev)
    lib.apply_dirichlet(A, flags_d, b_dev)
    torch.cuda.synchronize()
    nv.range_pop()
    nv.range_push("c2_factor")
    M.factor()
    torch.cuda.synchronize()
    nv.range_pop()
    nv.range_push("c2_spmv")
    for _ in range(3):
        A.spmv(1.0, b_dev, 0.0, y)
    torch.cuda.synchronize()
    nv.range_pop()
    nv.range_push("c2_ilu_apply")
    for _ in range(3):
        M.apply(b_dev, y)
    torch.cuda.synchronize()
    nv.range_pop()
    nv.range_push("c2_pcg")
    r.copy_(b_dev)
    lib.solve_pcg(A, M, r, x, tol=TOL, maxit=32)
    torch.cuda.synchronize()
    nv.range_pop()
    nv.range_push("c2_pcg_mixed")
    r.copy_(b_dev)
    lib.solve_pcg_mixed(A, M, r, x, tol=TOL, maxit=16)
    torch.cuda.synchronize()
    nv.range_pop()
    nv.range_push("c5")
    GZ.assemble_helmholtz(AZ, 2 * 3.1416 / 20, bz, load=loadz)
    MZ.factor()
    for _ in range(3):
        AZ.spmv(1.0, bz, 0.0, yz)
    for _ in range(3):
        MZ.apply(bz, yz)
    torch.cuda.synchronize()
    nv.range_pop()
    nv.range_push("c3_batch")
    B.solve(bb, xb, tol=TOL)
    torch.cuda.synchronize()
    nv.range_pop()
    nv.range_pop()
    log(f"[profile-run] c2 sweep mode {M.sweep}, lanes {A.lanes}, spmv kernel {A.spmv_kernel}; c5 sweep mode "
        f"{MZ.sweep}; c3 batch schedule {B.schedule}")


# ------------------------------------------------------- c1 and c5 sections
def build_c1(ctx, torch, dev):
    from delfem_b200 import lib, meshes
    m = meshes.unit_square_tri(256)
    G = lib.Mesh(ctx, m.coord, m.elem)
    rp, ci = G.pattern()
    A = lib.Matrix(ctx, rp, ci, 1)
    b = torch.empty(m.nnode, dtype=torch.float64, device=f"cuda:{dev}")
    G.assemble_poisson(A, 1.0, 1.0, b)
    fl = np.zeros(m.nnode, np.int32)
    fl[np.unique(m.bnd.ravel())] = 1
    lib.apply_dirichlet(A, torch.from_numpy(fl).cuda(dev), b)
    return A, b


def run_c1(ctx, torch, dev, timed, with_reference):
    """c1: 2-D Poisson 256^2 to rel.res 1e-10, plain FP64 and mixed, against the
    reference's own CPU solve of the same (bit-identical) system."""
    from delfem_b200 import lib
    A, b = build_c1(ctx, torch, dev)
    M = lib.ILU(A)
    M.factor()
    x = torch.zeros_like(b)
    r = b.clone()

    def plain():
        r.copy_(b)
        return lib.solve_pcg(A, M, r, x, tol=1e-10, maxit=20000)

    def mixed():
        r.copy_(b)
        return lib.solve_pcg_mixed(A, M, r, x, tol=1e-10, maxit=20000)

    plain()
    t_plain = timed(plain, 5)
    rc, it, conv = plain()
    x64 = x.cpu().numpy()
    mixed()
    t_mixed = timed(mixed, 5)
    rc_m, it_m, conv_m = mixed()
    xm = x.cpu().numpy()
    out = {"workload": "c1 2-D Poisson 256x256 P1 (N = 66,049), ILU(0) + PCG to rel.res 1e-10",
           "plain_s": t_plain, "iterations": it + 1, "mixed_s": t_mixed, "mixed_iterations": it_m + 1,
           "mixed_speedup_vs_plain": t_plain / t_mixed,
           "mixed_rel_err_vs_fp64": float(np.linalg.norm(xm - x64) / np.linalg.norm(x64)),
           "sweep_mode": M.sweep}
    if with_reference:
        try:
            from oracle import refshim as R
            d, o = A.get_values()
            rc_r, x_ref, it_r, conv_r, t_ilu, t_sol = R.mat_solve(A.N, 1, A.rowptr, A.colind, d, o,
                                                                  b.cpu().numpy(), R.PCG, 1e-10, 20000)
            out.update({"reference_cpu_s": t_ilu + t_sol, "reference_iterations": it_r + 1,
                        "rel_err_vs_reference": float(np.linalg.norm(x64 - x_ref) / np.linalg.norm(x_ref)),
                        "speedup_vs_reference_cpu": (t_ilu + t_sol) / t_plain})
        except Exception as e:  # the reference build may be absent
            out["reference_cpu_s"] = f"unavailable: {e}"
    for h in (M, A):
        h.close()
    return out


def run_c5(ctx, torch, dev, timed):
    """c5: Helmholtz k = 20 on the unit disk (~200k nodes), complex ILU(0)-COCG to
    rel.res 1e-8 in complex128 and with complex64 values inside complex128
    residual replacement.  The disk's nodes are numbered in horizontal bands
    (ILU level depth ~1200); numbered ring by ring, every row of the lower
    triangle would depend on the previous one and the sweeps would be a
    200k-step chain."""
    from delfem_b200 import lib, meshes
    m = meshes.unit_disk_tri(258, numbering="bands")
    G = lib.Mesh(ctx, m.coord, m.elem, m.bnd)
    rp, ci = G.pattern()
    A = lib.Matrix(ctx, rp, ci, 1, lib.COMPLEX)
    b = torch.empty(2 * m.nnode, dtype=torch.float64, device=f"cuda:{dev}")
    load = torch.from_numpy(meshes.gaussian_source_load(m).ravel()).cuda(dev)
    G.assemble_helmholtz(A, 2 * 3.1416 / 20, b, load=load)
    M = lib.ILU(A)
    M.factor()
    x = torch.zeros_like(b)
    r = b.clone()

    def plain():
        r.copy_(b)
        return lib.solve_pcocg(A, M, r, x, tol=1e-8, maxit=C5_MAXIT)

    def mixed():
        r.copy_(b)
        return lib.solve_pcocg_mixed(A, M, r, x, tol=1e-8, maxit=C5_MAXIT)

    plain()
    t_plain = timed(plain, 2)
    rc, it, conv = plain()
    x128 = x.clone()
    mixed()
    t_mixed = timed(mixed, 2)
    rc_m, it_m, conv_m = mixed()
    y = torch.empty_like(b)
    A.spmv(1.0, x, 0.0, y)
    torch.cuda.synchronize()
    res_m = float(torch.linalg.norm(b - y) / torch.linalg.norm(b))
    ref = reference_solution("c5")
    if ref is not None and int(ref["N"]) == A.N:
        xr = ref["x"]
        pick = lambda v: v.cpu().numpy().reshape(-1, 2)[ref["idx"]]  # noqa: E731
        ref_cmp = {"reference_iterations": int(ref["iters"]),
                   "complex128_rel_err_vs_reference": float(np.linalg.norm(pick(x128) - xr) / np.linalg.norm(xr)),
                   "complex64_rel_err_vs_reference": float(np.linalg.norm(pick(x) - xr) / np.linalg.norm(xr)),
                   "reference_sample": f"{ref['idx'].size} entries of the reference's Solve_PCOCG solution "
                                       f"(complex128, rel.res 1e-8)"}
    else:
        ref_cmp = {"reference": "fixture absent"}
    out = {"workload": f"c5 Helmholtz k=20 unit disk, {m.nnode} nodes (band numbering), complex ILU(0)-COCG to "
                       f"rel.res 1e-8", "sweep_mode": M.sweep,
           "complex128_s": t_plain, "iterations": it, "status": rc,
           "complex64_inner_s": t_mixed, "complex64_iterations": it_m, "complex64_status": rc_m,
           "complex64_speedup": t_plain / t_mixed, "complex64_true_rel_residual": res_m,
           "complex64_rel_err_vs_complex128": float(torch.linalg.norm(x - x128) / torch.linalg.norm(x128)),
           **ref_cmp}
    for h in (M, A, G):
        h.close()
    return out


def run_c4(torch, dev):
    """c4: the adjoint of 2-D plane-stress elasticity (128x128 grid of P1
    triangles, 2x2 blocks, nu = 0.3, per-element Young's modulus theta ~
    lognormal(0, 0.5), left edge clamped, traction (0, -1) on the right edge,
    L = 1/2 sum over 256 observed nodes |u - u_target|^2 with u_target from a
    second seeded theta).  One step = the forward solve (device assembly,
    elimination, ILU(0), PCG to 1e-12) and the backward (adjoint PCG with the
    same factorization, element kernel) through torch.autograd, timed on the
    host clock (the library synchronises).  Checked against an FP64 direct
    adjoint gradient and central finite differences (h = 1e-6) on 64 sampled
    elements, both FP64 on the host (tests/adjoint_ref.py)."""
    from delfem_b200 import adjoint, lib
    from tests import cases
    from tests.adjoint_ref import Reference
    ctx = lib.Context(dev)
    m, theta, theta_t, obs, fixed, load = cases.adjoint_case(128, seed=0)
    R = Reference(m.coord, m.elem, fixed, load, cases.LAM2_PS, cases.MYU2)
    ut = R.solve(theta_t)[1]
    idx = np.concatenate([2 * obs, 2 * obs + 1])
    prob = adjoint.PlaneStressProblem(ctx, m.coord, m.elem, fixed, load, cases.LAM2_PS, cases.MYU2, tol=1e-12)
    idx_t = torch.from_numpy(idx).cuda(dev)
    ut_t = torch.from_numpy(ut).cuda(dev)

    def step():
        prob._theta = None  # every step assembles and factors K(theta) again
        th = torch.tensor(theta, dtype=torch.float64, device=f"cuda:{dev}", requires_grad=True)
        u = adjoint.elastic_solve(th, prob)
        loss = 0.5 * torch.sum((u[idx_t] - ut_t[idx_t]) ** 2)
        loss.backward()
        return float(loss.item()), th.grad

    step()
    ts = []
    for _ in range(5):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss, g = step()
        torch.cuda.synchronize()
        ts.append(time.perf_counter() - t0)
    g_dev = g.cpu().numpy()

    def gfun(uu):
        gg = np.zeros_like(uu)
        gg[idx] = uu[idx] - ut[idx]
        return 0.5 * np.sum((uu[idx] - ut[idx]) ** 2), gg

    t0 = time.perf_counter()
    L_ref, g_ref = R.grad(theta, gfun)
    elems = np.random.default_rng(100).choice(m.elem.shape[0], 64, replace=False)
    fd = R.fd(theta, idx, ut, elems, h=1e-6)
    t_check = time.perf_counter() - t0
    ctx.close()
    return {"workload": "c4 plane-stress adjoint 128x128 P1 (N = 16,641, b = 2, 32,768 elements), 256 observed "
                        "nodes, forward + backward per step",
            "forward_backward_s": statistics.median(ts), "forward_iterations": prob.last_iters + 1,
            "loss": loss, "loss_rel_err_vs_fp64": abs(loss - L_ref) / abs(L_ref),
            "grad_rel_err_vs_fp64_adjoint": float(np.linalg.norm(g_dev - g_ref) / np.linalg.norm(g_ref)),
            "grad_rel_err_vs_central_fd": float(np.linalg.norm(g_dev[elems] - fd) / np.linalg.norm(fd)),
            "fd": "central differences, h = 1e-6, 64 sampled elements, FP64 direct solves on the host",
            "host_check_s": t_check}


# -------------------------------------------------------------------- our arm
def run_ours(args, rank, world):
    import torch
    from delfem_b200 import lib
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    ctx = lib.Context(dev)
    lib.check(lib.lib().dfm_ctx_set_stream(ctx.h, lib.C.c_void_p(stream.cuda_stream)))
    m, G, A, b_dev, t_asm = build_c2(ctx, torch, dev)
    N, b, ncrs = A.N, A.b, A.ncrs
    assert (N, b, ncrs) == (C2_CONFIG["N"], C2_CONFIG["b"], C2_CONFIG["ncrs"])
    M = lib.ILU(A)
    # range-sweep CTAs as patches across the beam's long axis (the autotuner
    # times this partition beside balanced ranges of the natural order)
    part, nparts = lib.sweep_partition_patches(m.coord, torch.cuda.get_device_properties(dev).multi_processor_count)
    M.set_sweep_partition(part, nparts)
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
    x64 = x.clone()

    def timed(fn, reps):
        out = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            out.append(e0.elapsed_time(e1) / 1e3)
        return statistics.median(out)

    def true_rel_residual(xv):
        y = torch.empty_like(b_dev)
        A.spmv(1.0, xv, 0.0, y)
        torch.cuda.synchronize()
        return float(torch.linalg.norm(b_dev - y) / torch.linalg.norm(b_dev))

    rr = true_rel_residual(x64)

    # ---- parity at scale: the c2 solve to 1e-10 against the reference's own x ----
    parity = {}
    ref = reference_solution("c2")
    if ref is not None and rank == 0:
        x10 = torch.zeros_like(b_dev)
        r.copy_(b_dev)
        rc10, it10, conv10 = lib.solve_pcg(A, M, r, x10, tol=1e-10, maxit=20000)
        xh = x10.cpu().numpy()
        parity = {"tol": 1e-10, "iterations": it10 + 1, "reference_iterations": int(ref["iters"]) + 1,
                  "rel_err_vs_reference_sampled": float(np.linalg.norm(xh[ref["idx"]] - ref["x"]) /
                                                        np.linalg.norm(ref["x"])),
                  "rel_norm_diff_vs_reference": float(abs(np.linalg.norm(xh) - float(ref["xnorm"])) /
                                                      float(ref["xnorm"])),
                  "sample": f"{ref['idx'].size} entries (every {int(ref['idx'][1])}th DOF) of the reference's "
                            f"Solve_PCG solution, and its 2-norm",
                  "true_rel_residual": true_rel_residual(x10)}
        log(f"[bench] c2 at 1e-10: {it10 + 1} iterations (reference {int(ref['iters']) + 1}), rel err vs the "
            f"reference's x {parity['rel_err_vs_reference_sampled']:.2e}")

    # ---- kernel breakdown (CUDA events on the library stream) ----
    y = torch.empty_like(b_dev)
    t_spmv = A.time_spmv(x, y, 50)
    t_apply = M.time_apply(r, y, 20)
    M0 = lib.ILU(A)  # the same preconditioner with balanced ranges of the natural order only
    M0.factor()
    t_apply_nat = M0.time_apply(r, y, 20)
    sweep_nat = M0.sweep
    M0.close()
    t_factor = timed(lambda: M.factor(), 3)
    B_spmv, B_ilu, B_it = alg_bytes(N, ncrs, b)
    peaks_p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peaks = json.load(open(peaks_p)) if os.path.exists(peaks_p) else {}
    hbm = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if peaks else "fallback"
    n_it = iters + 1
    t_iter = (t_step - t_factor) / n_it
    share_sweep = t_apply * n_it / t_step
    share_spmv = t_spmv * n_it / t_step
    kernels = {
        "spmv_bcrs_b3": {"ms": t_spmv * 1e3, "alg_bytes": B_spmv, "gbs": B_spmv / t_spmv / 1e9,
                         "frac": B_spmv / t_spmv / 1e9 / hbm, "share_of_step": share_spmv,
                         "kernel": A.spmv_kernel, "lanes": A.lanes},
        "ilu0_fwd_bwd": {"ms": t_apply * 1e3, "alg_bytes": B_ilu, "gbs": B_ilu / t_apply / 1e9,
                         "frac": B_ilu / t_apply / 1e9 / hbm, "share_of_step": share_sweep,
                         "sweep_mode": M.sweep, "partition_parts": nparts,
                         "ms_without_partition": t_apply_nat * 1e3, "sweep_mode_without_partition": sweep_nat},
        "ilu0_factor": {"ms": t_factor * 1e3},
        "pcg_iteration": {"ms": t_iter * 1e3, "alg_bytes": B_it, "gbs": B_it / t_iter / 1e9},
        "assembly_c2": {"ms": t_asm * 1e3},
    }
    dom = "ilu0_fwd_bwd" if share_sweep >= share_spmv else "spmv_bcrs_b3"
    dk = kernels[dom]
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp)).get(dom)

    # ---- mixed precision on the same system ----
    mixed = {}
    if not args.skip_mixed:
        xm = torch.zeros_like(b_dev)

        def mstep():
            M.factor()
            r.copy_(b_dev)
            torch.cuda.synchronize()
            return lib.solve_pcg_mixed(A, M, r, xm, tol=TOL, maxit=40000)

        mstep()
        t_mixed = timed(mstep, max(2, min(args.steps, 3)))
        rc_m, it_m, conv_m = mstep()
        mixed = {"solve_s": t_mixed, "plain_fp64_solve_s": t_step, "speedup_vs_plain": t_step / t_mixed,
                 "iterations": it_m + 1, "plain_iterations": n_it, "status": rc_m,
                 "true_rel_residual": true_rel_residual(xm),
                 "rel_err_vs_fp64_solution": float(torch.linalg.norm(xm - x64) / torch.linalg.norm(x64))}

    # ---- ILU(1) on the same system (SetFillInLevel(1), the reference's default for solids) ----
    iluk = {}
    if not args.skip_iluk and world == 1:
        t0 = time.perf_counter()
        M1 = lib.ILU(A, fill_level=1)
        t_sym = time.perf_counter() - t0
        M1.set_sweep_partition(part, nparts)  # the same patches as the ILU(0) solve
        x1 = torch.zeros_like(b_dev)

        def k1step():
            M1.factor()
            r.copy_(b_dev)
            torch.cuda.synchronize()
            return lib.solve_pcg(A, M1, r, x1, tol=TOL, maxit=20000)

        k1step()
        t_k1 = timed(k1step, max(2, min(args.steps, 3)))
        rc_k, it_k, conv_k = k1step()
        t_k1_apply = M1.time_apply(r, y, 10)
        iluk = {"fill_level": 1, "factor_ncrs": M1.ncrs, "matrix_ncrs": ncrs, "symbolic_s": t_sym,
                "solve_s": t_k1, "iterations": it_k + 1, "status": rc_k, "apply_ms": t_k1_apply * 1e3,
                "sweep_mode": M1.sweep, "ilu0_solve_s": t_step, "ilu0_iterations": n_it,
                "speedup_vs_ilu0": t_step / t_k1, "true_rel_residual": true_rel_residual(x1),
                "rel_err_vs_ilu0_solution": float(torch.linalg.norm(x1 - x64) / torch.linalg.norm(x64))}
        M1.close()
        log(f"[bench] c2 ILU(1): factor ncrs {M1.ncrs} (A {ncrs}), {it_k + 1} iterations, {t_k1:.3f}s "
            f"(ILU(0): {n_it}, {t_step:.3f}s)")

    # ---- end-to-end through the C ABI with host buffers ----
    diag_d, off_d = A.get_values()
    diag_h = torch.from_numpy(diag_d).pin_memory()
    off_h = torch.from_numpy(off_d).pin_memory()
    b_h = b_dev.cpu().pin_memory()
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
    h2d = diag_h.numel() * 8 + off_h.numel() * 8 + b_h.numel() * 8
    d2h = x_h.numel() * 8

    # ---- c3 batched vs looped ----
    batched = {}
    if not args.skip_batched and world == 1:
        batched = run_c3(ctx, torch, dev, stream, timed, args.steps)
    elif not args.skip_batched:
        batched = {"sharded": run_c3_sharded(torch, dev, stream, args.steps)}
    c1 = {}
    c4 = {}
    c5 = {}
    if not args.skip_extra and world == 1:
        c1 = run_c1(ctx, torch, dev, timed, rank == 0 and not args.no_cpu_baseline)
        c4 = run_c4(torch, dev)
        c5 = run_c5(ctx, torch, dev, timed)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            n_full = reference_runs().get("c2", {}).get(f"tol{TOL:g}", {}).get("iterations") or n_it
            t_ilu, t_iter_ref = cpu_reference_sample(N, b, A.rowptr, A.colind, diag_d, off_d, b_h.numpy(), 30)
            v = 1.0 / (t_ilu + n_full * t_iter_ref)
            cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"the reference's ILU(0) ({t_ilu:.2f}s) + 30 Solve_PCG iterations "
                             f"({t_iter_ref * 1e3:.1f} ms/it) on one host core (single-threaded code), "
                             f"scaled to its {n_full} iterations to 1e-8",
                   "t_ilu_s": t_ilu, "t_iter_s": t_iter_ref, "iterations": n_full}
        except Exception as e:  # the reference build may be absent
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": f"unavailable: {e}"}

    launches = 2 + 4 + 16 * ((n_it + 15) // 16) * 5
    if rank == 0:
        line = {
            "metric": METRIC, "value": world / t_step, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(C2_CONFIG, parallelism=f"replicas x{world}"),
            "iterations": n_it, "conv": conv, "true_rel_residual": rr, "solve_time_s": t_step,
            "parity_c2_1e-10": parity,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": dk["gbs"], "peak": hbm, "unit": "GB/s",
                         "frac": dk["frac"], "traffic": traffic, "peak_source": peak_src},
            "spmv_roofline": {"achieved": kernels["spmv_bcrs_b3"]["gbs"], "peak": hbm, "unit": "GB/s",
                              "frac": kernels["spmv_bcrs_b3"]["frac"]},
            "kernels": kernels,
            "mixed": mixed,
            "ilu1": iluk,
            "batched": batched,
            "c1": c1,
            "c4": c4,
            "c5": c5,
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
    ap.add_argument("--skip-batched", action="store_true")
    ap.add_argument("--skip-mixed", action="store_true")
    ap.add_argument("--skip-iluk", action="store_true", help="skip the c2 ILU(1) section")
    ap.add_argument("--skip-extra", action="store_true", help="skip the c1 and c5 sections")
    ap.add_argument("--profile-run", action="store_true")
    args = ap.parse_args()
    if args.profile_run:
        run_profile()
        return
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
