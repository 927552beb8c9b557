"""The resident server: jobs of uneven size submitted together run
concurrently and in merged batches; each result equals the same job gridded
alone (and the FP64 oracle), the HBM budget is respected, and a job that can
never fit is rejected."""
import time

import numpy as np
import pytest
import torch

import fpga_gridding_b200 as fg
from fpga_gridding_b200 import _lib, workloads as W
from fpga_gridding_b200.serving import Server
from oracle.oracle import rel_rms

pytestmark = pytest.mark.gpu


def _jobs():
    wls = W.batch_channels(seed=9, num_channels=6, num_stations=40,
                           num_times=24, grid_size=512, num_w_planes=12)
    wls += [W.plain_small(seed=10 + i, num_stations=24 + 8 * i, num_times=30,
                          grid_size=256 * (1 + i % 2), num_w_planes=8)
            for i in range(4)]
    out = []
    for w in wls:
        w32 = w.to(dtype=torch.float32, device="cuda")
        out.append(dict(wl=w, uu=w32.uu, vv=w32.vv, ww=w32.ww, vis=w32.vis,
                        weight=w32.weight,
                        cell=float(np.float32(w.cell_size_rad)),
                        wsc=float(np.float32(w.w_scale)), g=w.grid_size))
    return out


def _oracle_grid(oracle, w):
    d = w.numpy()
    for k in ("conv_func", "uu", "vv", "ww", "vis", "weight"):
        d[k] = np.asarray(d[k], np.float32).astype(np.float64)
    d["cell_size_rad"] = float(np.float32(d["cell_size_rad"]))
    d["w_scale"] = float(np.float32(d["w_scale"]))
    return oracle.grid_d(d, threads=8)


def _collect(srv, n, deadline_s=300.0):
    """Every completion of n jobs; fails the test (instead of polling
    forever) if they have not all arrived within deadline_s."""
    done = {}
    t_end = time.monotonic() + deadline_s
    while len(done) < n:
        assert time.monotonic() < t_end, \
            f"{n - len(done)} of {n} jobs not completed after {deadline_s} s"
        for c in srv.poll(timeout=1.0):
            done[c["tag"]] = c
    return done


def test_mix_equals_alone_and_oracle(oracle):
    jobs = _jobs()
    ws = fg.Workspace(0)
    cubes = [fg.Cube(ws, j["wl"].support, j["wl"].oversample,
                     j["wl"].conv_size_half,
                     np.asarray(j["wl"].conv_func, np.float32),
                     data_is_double=False) for j in jobs]
    srv = Server(0, budget_bytes=8 << 30, slots=3, max_batch=4)
    for t, (j, c) in enumerate(zip(jobs, cubes)):
        srv.submit(t, c, j["uu"], j["vv"], j["ww"], j["vis"], j["weight"],
                   j["cell"], j["wsc"], j["g"])
    done = _collect(srv, len(jobs))
    assert max(c["batch_size"] for c in done.values()) > 1   # merged launches
    for t, (j, c) in enumerate(zip(jobs, cubes)):
        comp = done[t]
        assert comp["status"] == 0
        mix = srv.grid(comp).cpu().numpy()
        alone = torch.zeros(2 * j["g"] ** 2, device="cuda")
        skip = torch.zeros(1, dtype=torch.int64, device="cuda")
        norm = torch.zeros(1, dtype=torch.float64, device="cuda")
        fg.grid_device(ws, c, j["uu"], j["vv"], j["ww"], j["vis"],
                       j["weight"], j["cell"], j["wsc"], j["g"], alone, skip,
                       norm)
        torch.cuda.synchronize()
        sk, nrm, ref = _oracle_grid(oracle, j["wl"])
        assert comp["num_skipped"] == int(skip.item()) == sk
        # a merged launch splits the norm reduction differently
        assert abs(comp["norm"] - norm.item()) <= 1e-13 * abs(nrm)
        assert abs(comp["norm"] - nrm) <= 1e-12 * abs(nrm)
        assert rel_rms(mix, alone.cpu().numpy()) <= 2e-6
        assert rel_rms(mix, ref) <= 1e-5
        assert comp["submit_s"] <= comp["start_s"] <= comp["end_s"]
        srv.release(t)
    srv.close()
    for c in cubes:
        c.close()
    ws.close()


def test_budget_is_respected_and_impossible_job_rejected():
    jobs = _jobs()[:5]
    ws = fg.Workspace(0)
    cubes = [fg.Cube(ws, j["wl"].support, j["wl"].oversample,
                     j["wl"].conv_size_half,
                     np.asarray(j["wl"].conv_func, np.float32),
                     data_is_double=False) for j in jobs]
    # room for about one small job at a time
    budget = 64 << 20
    srv = Server(0, budget_bytes=budget, slots=4, max_batch=8)
    for t, (j, c) in enumerate(zip(jobs, cubes)):
        srv.submit(t, c, j["uu"], j["vv"], j["ww"], j["vis"], j["weight"],
                   j["cell"], j["wsc"], j["g"])
    # a 8192^2 grid (512 MB) can never fit a 64 MB budget
    j = jobs[0]
    srv.submit(99, cubes[0], j["uu"], j["vv"], j["ww"], j["vis"],
               j["weight"], j["cell"], j["wsc"], 8192)
    done = {}
    t_end = time.monotonic() + 300.0
    while len(done) < len(jobs) + 1:
        assert time.monotonic() < t_end, "jobs not completed after 300 s"
        for c in srv.poll(timeout=1.0):
            done[c["tag"]] = c
            used, cap = srv.memory()
            assert used <= cap
            if c["status"] == 0:
                srv.release(c["tag"])
    assert done[99]["status"] == _lib.ERR_OVER_BUDGET
    assert all(done[t]["status"] == 0 for t in range(len(jobs)))
    srv.close()
    for c in cubes:
        c.close()
    ws.close()


def test_time_sliced_large_job_and_reserved_small_slot():
    """A job of about 8.9 million visibilities (above the server's
    small-batch and slice sizes, so its gridding runs as several
    time-sliced launches) submitted with small jobs, which the reserved
    small-job slot takes past it on the high-priority stream: every result
    equals the same job gridded alone."""
    big = W.plain_small(seed=21, num_stations=128, num_times=1100,
                        grid_size=1024, num_w_planes=16)
    assert big.num_points > 8_000_000
    small = _jobs()[:3]
    b32 = big.to(dtype=torch.float32, device="cuda")
    jobs = [dict(wl=big, uu=b32.uu, vv=b32.vv, ww=b32.ww, vis=b32.vis,
                 weight=b32.weight, cell=float(np.float32(big.cell_size_rad)),
                 wsc=float(np.float32(big.w_scale)), g=big.grid_size)] + small
    ws = fg.Workspace(0)
    cubes = [fg.Cube(ws, j["wl"].support, j["wl"].oversample,
                     j["wl"].conv_size_half,
                     np.asarray(j["wl"].conv_func, np.float32),
                     data_is_double=False) for j in jobs]
    srv = Server(0, budget_bytes=16 << 30, slots=3, max_batch=4)
    for t, (j, c) in enumerate(zip(jobs, cubes)):
        srv.submit(t, c, j["uu"], j["vv"], j["ww"], j["vis"], j["weight"],
                   j["cell"], j["wsc"], j["g"])
    done = _collect(srv, len(jobs))
    for t, (j, c) in enumerate(zip(jobs, cubes)):
        comp = done[t]
        assert comp["status"] == 0
        mix = srv.grid(comp).cpu().numpy()
        alone = torch.zeros(2 * j["g"] ** 2, device="cuda")
        skip = torch.zeros(1, dtype=torch.int64, device="cuda")
        norm = torch.zeros(1, dtype=torch.float64, device="cuda")
        fg.grid_device(ws, c, j["uu"], j["vv"], j["ww"], j["vis"],
                       j["weight"], j["cell"], j["wsc"], j["g"], alone, skip,
                       norm)
        torch.cuda.synchronize()
        assert comp["num_skipped"] == int(skip.item())
        assert abs(comp["norm"] - norm.item()) <= 1e-13 * abs(norm.item())
        assert rel_rms(mix, alone.cpu().numpy()) <= 2e-6
        srv.release(t)
    srv.close()
    for c in cubes:
        c.close()
    ws.close()
