"""The N>1 path of bench.py: independent replicas, one per rank, with no data-path collective.

Two gloo ranks on the CPU stand in for two GPUs: the replica aggregation must take the maximum of
the ranks' device times and the sum of their processed cells, and under torchrun the reference arm
runs on rank 0 only (the other ranks exit 0 without work).
"""
import os
import socket
import subprocess
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as td
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        times = np.array([10.0 + rank, 5.0 - rank, 3.0 * (rank + 1), 20.0 + 2 * rank])
        cells = np.array([1000.0 * (rank + 1), 100.0 * (rank + 1)])
        t, c = bench.reduce_over_ranks(times, cells, "cpu")
        out[rank] = (t.tolist(), c.tolist())
        td.barrier()
    finally:
        td.destroy_process_group()


def test_replica_reduction_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    for r in range(world):
        t, c = res[r]
        assert t == [11.0, 5.0, 6.0, 22.0]  # max over ranks
        assert c == [3000.0, 300.0]         # sum over ranks


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def _rank_dies(rank, world, port, out):
    import datetime

    import torch.distributed as td
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        os._exit(3)  # this replica dies before the reduction
    import time
    t0 = time.time()
    try:
        bench.reduce_over_ranks(np.ones(4), np.ones(2), "cpu")
        out[rank] = "no error"
    except Exception as e:  # the survivor sees an error instead of waiting for ever
        out[rank] = f"error after {time.time() - t0:.1f}s: {type(e).__name__}"
    os._exit(0)


def test_a_dead_replica_makes_the_reduction_fail_not_hang():
    world = 2
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_dies, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        alive = [p for p in procs if p.is_alive()]
        for p in alive:
            p.kill()
        assert not alive, "a rank hung"
        res = dict(out)
    assert res.get(0, "").startswith("error after"), res
