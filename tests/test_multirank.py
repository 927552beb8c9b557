"""The replica (multi-GPU) host logic on CPU with gloo, world size 2: each
rank grids its own independent job, the step time is the max over ranks and
the throughput counts every rank's points."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from fpga_gridding_b200 import replicas, workloads as W
        w, r, _ = replicas.rank_info()
        assert (w, r) == (world, rank)
        wl = W.plain_large(seed=replicas.replica_seed(1, rank),
                           num_stations=8, num_times=4, grid_size=256,
                           num_w_planes=4)
        # per-rank elapsed time differs; the job time is the slowest
        elapsed = 1.0 + rank
        worst = replicas.max_over_ranks(elapsed, world)
        thr = replicas.weak_scaling_throughput(wl.num_points, 3, elapsed,
                                               world)
        out[rank] = (float(wl.uu[:4].sum()), worst, thr, wl.num_points)
    finally:
        dist.destroy_process_group()


def test_two_replicas_gloo():
    mp_ctx = mp.get_context("spawn")
    manager = mp_ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [mp_ctx.Process(target=_worker, args=(r, 2, port, out))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    (u0, w0, t0, n0), (u1, w1, t1, n1) = out[0], out[1]
    assert u0 != u1                      # independent jobs per rank
    assert w0 == w1 == 2.0               # max over ranks
    assert t0 == t1 == pytest.approx((n0 + n1) * 3 / 2.0)


def test_single_rank_is_identity():
    from fpga_gridding_b200 import replicas
    assert replicas.max_over_ranks(3.5, 1) == 3.5
    assert replicas.weak_scaling_throughput(10, 2, 4.0, 1) == 5.0
