"""The multi-GPU path of this SPM step is replicas only: every rank advances
its own box and the only communication is the barrier and the max-over-ranks
timing reduction of bench.py.  This runs that host logic with two gloo ranks
on the CPU, each rank advancing its own oracle box."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    import bench
    from oracle import spm, udf

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    cfg = udf.ns_config((4, 4, 4), 1, seed=10 + rank, kbt=1e-3)
    o = spm.SpmOracle(cfg)
    dist.barrier()
    o.run(2)
    elapsed = 1.0 + rank  # a stand-in per-rank time: rank 1 is the slowest
    mx = bench.reduce_max(elapsed, dist, device="cpu")
    value = bench.replica_value(2, world, mx)
    dist.barrier()
    out[rank] = (mx, value, float(np.abs(o.p.x).sum()))
    dist.destroy_process_group()


def test_two_gloo_replicas_reduce_max():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] == 2.0          # both ranks see the slowest rank's time
    assert out[0][1] == out[1][1] == 2 * world / 2.0  # all ranks' steps over the max time
    assert out[0][2] != out[1][2]                  # the replicas advanced different boxes


def _worker_fail(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    dist.barrier()
    if rank == 1:
        # a replica that fails between steps: it leaves without taking part in
        # the timing reduction
        os._exit(3)
    try:
        bench.reduce_max(1.0, dist, device="cpu")
        out[rank] = "completed"
    except Exception as e:  # the short process-group timeout ends the wait
        out[rank] = f"error: {type(e).__name__}"
    os._exit(0)


def test_failed_replica_ends_the_others_wait_with_an_error():
    """Failure detection on the host: when one replica exits between steps,
    the surviving rank's next collective (the max-over-ranks reduction of the
    timing) ends with an error after the process group's short timeout
    instead of waiting forever."""
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker_fail, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert procs[1].exitcode == 3
    assert procs[0].exitcode == 0
    assert str(out.get(0, "")).startswith("error"), out.get(0)
