"""Sharding of batched instances over ranks: the greedy partition (pure host
logic) and the gather of per-instance results across two gloo ranks on the
CPU, with instances solved by the oracle in the ranks (the GPU batch is the
product's solve_local; here a CPU stand-in exercises the plumbing)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from delfem_b200 import shard


def test_partition_covers_all_and_balances():
    rng = np.random.default_rng(0)
    n = np.rint(np.exp(rng.uniform(np.log(32), np.log(512), 512))).astype(int)
    work = (n + 1.0) ** 2
    for world in (1, 2, 3, 8):
        parts = shard.partition(work, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(512))
        ld = shard.loads(work, parts)
        # LPT bound: max load <= mean + largest item
        assert ld.max() <= ld.mean() + work.max() + 1e-9
        assert parts == shard.partition(work, world)  # deterministic


def test_partition_edge_cases():
    assert shard.partition([], 3) == [[], [], []]
    assert shard.partition([5.0], 2) == [[0], []]
    assert shard.partition([1, 1, 1, 1], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        shard.partition([1.0], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, sizes, out_path):
    import datetime

    import torch.distributed as dist

    from delfem_b200 import meshes
    from oracle import port as P
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))

    def solve_local(insts):
        res = []
        for n in insts:
            m = meshes.unit_square_tri(int(n))
            S = P.System(*P.pattern(m.nnode, m.elem), 1)
            S.asm_poisson(m, 1.0, 1.0)
            S.apply_bc(P.bc_flags_from_bnd(m.nnode, 1, m.bnd))
            ns, fd, fo = S.ilu0()
            o = S.solve(fd, fo, tol=1e-10, maxit=1000)
            res.append((rank, int(n), o["iters"], float(o["x"].max())))
        return res

    out = shard.solve_sharded(list(sizes), [(n + 1) ** 2 for n in sizes], solve_local)
    if rank == 0:
        np.save(out_path, np.array([(r, n, it, xm) for r, n, it, xm in out], dtype=np.float64))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_solve_gathers_in_order_over_two_gloo_ranks(tmp_path):
    sizes = [12, 4, 20, 7, 16, 9, 3]
    out_path = str(tmp_path / "out.npy")
    mp.spawn(_worker, args=(2, _free_port(), sizes, out_path), nprocs=2, join=True)
    got = np.load(out_path)
    assert got.shape == (len(sizes), 4)
    assert list(got[:, 1].astype(int)) == sizes          # original order restored
    parts = shard.partition([(n + 1) ** 2 for n in sizes], 2)
    for r, p in enumerate(parts):                        # each instance solved by its owner
        assert all(int(got[k, 0]) == r for k in p)
    assert set(got[:, 0].astype(int)) == {0, 1}
    # results equal a single-process solve
    from delfem_b200 import meshes
    from oracle import port as P
    for k, n in enumerate(sizes):
        m = meshes.unit_square_tri(n)
        S = P.System(*P.pattern(m.nnode, m.elem), 1)
        S.asm_poisson(m, 1.0, 1.0)
        S.apply_bc(P.bc_flags_from_bnd(m.nnode, 1, m.bnd))
        ns, fd, fo = S.ilu0()
        o = S.solve(fd, fo, tol=1e-10, maxit=1000)
        assert got[k, 2] == o["iters"] and got[k, 3] == o["x"].max()


def _timed_worker(rank, world, port, sizes, out_path):
    import datetime
    import time as _t

    import torch.distributed as dist

    from delfem_b200 import meshes
    from oracle import port as P
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))

    def solve_local(idx):
        t0 = _t.perf_counter()
        res = []
        for k in idx:
            m = meshes.unit_square_tri(int(sizes[k]))
            S = P.System(*P.pattern(m.nnode, m.elem), 1)
            S.asm_poisson(m, 1.0, 1.0)
            S.apply_bc(P.bc_flags_from_bnd(m.nnode, 1, m.bnd))
            ns, fd, fo = S.ilu0()
            o = S.solve(fd, fo, tol=1e-10, maxit=1000)
            res.append((rank, o["iters"]))
        return _t.perf_counter() - t0 + 0.01 * (rank + 1), res  # a rank-dependent time to check the max

    out = shard.timed_sharded([(n + 1) ** 2 for n in sizes], solve_local)
    if rank == 0:
        np.save(out_path, np.array([out["seconds"], *out["per_rank_seconds"], *out["per_rank_instances"]] +
                                   [v for r in out["results"] for v in r], dtype=np.float64))
    dist.barrier()
    dist.destroy_process_group()


def test_timed_sharded_max_over_two_gloo_ranks(tmp_path):
    """The bench's sharded batch (bench.py at --gpus N): per-rank shares, the
    job time as the max over ranks, per-instance results gathered in order."""
    sizes = [10, 3, 14, 6, 8]
    out_path = str(tmp_path / "t.npy")
    mp.spawn(_timed_worker, args=(2, _free_port(), sizes, out_path), nprocs=2, join=True)
    v = np.load(out_path)
    t_max, t0, t1, n0, n1 = v[:5]
    assert t_max == max(t0, t1) and t1 >= 0.02
    parts = shard.partition([(n + 1) ** 2 for n in sizes], 2)
    assert (n0, n1) == (len(parts[0]), len(parts[1])) and n0 + n1 == len(sizes)
    res = v[5:].reshape(-1, 2)
    for r, p in enumerate(parts):
        assert all(int(res[k, 0]) == r for k in p)
    assert all(res[:, 1] > 0)
