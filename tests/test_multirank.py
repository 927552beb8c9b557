"""The replica (multi-GPU) host logic on CPU with gloo, world size 2: each
rank builds and grids its own independent job (the CPU oracle standing in
for the rank's GPU), the step time is the max over ranks, the throughput
counts every rank's points, and the gathered per-rank results equal each
replica gridded alone."""
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
        # The rank grids its own replica (the CPU oracle stands in for the
        # rank's GPU here) and every rank's result summary is gathered:
        # no collective touches the grids themselves.
        from oracle import oracle as O
        skipped, norm, grid = O.grid_d(wl.numpy())
        mine = torch.tensor([float(skipped), norm,
                             float(abs(grid).sum())], dtype=torch.float64)
        every = [torch.zeros(3, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(every, mine)
        out[rank] = (float(wl.uu[:4].sum()), worst, thr, wl.num_points,
                     [t.tolist() for t in every])
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
    (u0, w0, t0, n0, g0), (u1, w1, t1, n1, g1) = out[0], out[1]
    assert u0 != u1                      # independent jobs per rank
    assert w0 == w1 == 2.0               # max over ranks
    assert t0 == t1 == pytest.approx((n0 + n1) * 3 / 2.0)
    # each rank's grid is its own replica gridded alone, bit for bit, and
    # both ranks see the same gathered summaries
    from fpga_gridding_b200 import replicas, workloads as W
    from oracle import oracle as O
    assert g0 == g1
    for rank in range(2):
        wl = W.plain_large(seed=replicas.replica_seed(1, rank),
                           num_stations=8, num_times=4, grid_size=256,
                           num_w_planes=4)
        skipped, norm, grid = O.grid_d(wl.numpy())
        assert g0[rank] == [float(skipped), norm, float(abs(grid).sum())]
    assert g0[0] != g0[1]


def test_single_rank_is_identity():
    from fpga_gridding_b200 import replicas
    assert replicas.max_over_ranks(3.5, 1) == 3.5
    assert replicas.weak_scaling_throughput(10, 2, 4.0, 1) == 5.0
