"""The multi-GPU path of bench.py is replicas (one per rank, no data-path collective); its only
cross-rank steps are the barrier and the max-over-ranks job time. Checked here with two gloo ranks
on CPU: every rank gets the slowest rank's time, the job rate counts all ranks' units, and the
reference arm prints on rank 0 only."""

import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        torch.distributed.barrier()
        mine = [10.0 + rank, 20.0 - rank]
        got = bench.max_over_ranks(torch, mine, world, "cpu")
        out.put((rank, got, bench.job_rate(100, world, got[0])))
    finally:
        torch.distributed.destroy_process_group()


def test_max_over_ranks_and_job_rate_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, rate in res:
        assert got == [11.0, 20.0]               # the slowest rank's time, on every rank
        assert abs(rate - 100 * 2 / 11e-3) < 1e-6  # units of both replicas over that time


def test_reference_arm_rank1_prints_nothing():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "3", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def _serve_partition(rank, world, port, q):
    """One replica: the maps whose index is rank mod world, served by this rank's router."""
    import numpy as np
    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    bench._package()  # registers h2factory_b200 in this spawned process
    from h2factory_b200.serving import DenseExecutor, MatvecServer, ReplicaRouter

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    rng = np.random.default_rng(0)
    maps = [rng.standard_normal((30 + 5 * i, 30 + 5 * i)) for i in range(6)]  # same on every rank
    mine = [i for i in range(len(maps)) if i % world == rank]
    router = ReplicaRouter([MatvecServer(DenseExecutor(), budget_bytes=1e9, max_block=4, slots=1)])
    for i in mine:
        router.add_map(i, maps[i])
    ok = 0
    for i in mine:
        x = np.ones(maps[i].shape[0])
        ok += int(np.allclose(router.submit(i, x).result(timeout=30), maps[i] @ x))
    router.close()
    served = torch.tensor([float(ok)])
    dist.all_reduce(served)  # host-side count only; the products themselves never cross ranks
    q.put((rank, sorted(mine), float(served.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_maps_partitioned_across_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_serve_partition, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == [0, 2, 4] and res[1][1] == [1, 3, 5]  # a partition of the maps
    assert res[0][2] == res[1][2] == 6.0                      # every map served exactly once
