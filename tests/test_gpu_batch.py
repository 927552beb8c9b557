"""Batched gridding: many jobs with uneven sizes, their own cubes and grids,
in one sort and one persistent gridding launch.  Each job's result must
equal the same job gridded alone and the FP64 oracle."""
import numpy as np
import pytest
import torch

import fpga_gridding_b200 as fg
from fpga_gridding_b200 import _lib, workloads as W
from oracle.oracle import rel_rms

pytestmark = pytest.mark.gpu


def _dev(t, dtype):
    return t.to(device="cuda", dtype=dtype).contiguous()


def _jobs(single):
    real = torch.float32 if single else torch.float64
    wls = W.batch_channels(seed=5, num_channels=5, num_stations=48,
                           num_times=30, grid_size=512, num_w_planes=16)
    wls.append(W.plain_small(seed=4, num_stations=32, num_times=40,
                             grid_size=256, num_w_planes=8))
    # an empty job in the middle
    wls.insert(2, wls[0].subset(slice(0, 0)))
    return [w.to(dtype=real) for w in wls]


def _oracle(oracle, w, single):
    d = w.numpy()
    if single:
        for k in ("conv_func", "uu", "vv", "ww", "vis", "weight"):
            d[k] = np.asarray(d[k], np.float32).astype(np.float64)
        d["cell_size_rad"] = float(np.float32(d["cell_size_rad"]))
        d["w_scale"] = float(np.float32(d["w_scale"]))
    return oracle.grid_d(d, threads=8)


@pytest.mark.parametrize("single,accum", [(True, _lib.ACCUM_PLAIN),
                                          (True, _lib.ACCUM_COMPENSATED),
                                          (False, _lib.ACCUM_PLAIN)])
def test_batch_matches_solo_and_oracle(oracle, single, accum):
    wls = _jobs(single)
    real = torch.float32 if single else torch.float64
    ws = fg.Workspace(0)
    cubes = [fg.Cube(ws, w.support, w.oversample, w.conv_size_half,
                     w.conv_func, data_is_double=not single) for w in wls]

    def scal(w):
        if single:
            return float(np.float32(w.cell_size_rad)), float(np.float32(w.w_scale))
        return w.cell_size_rad, w.w_scale

    def job(w, cube):
        cell, wsc = scal(w)
        return dict(cube=cube, uu=_dev(w.uu, real), vv=_dev(w.vv, real),
                    ww=_dev(w.ww, real), vis=_dev(w.vis, real),
                    weight=_dev(w.weight, real), cell_size_rad=cell,
                    w_scale=wsc, grid_size=w.grid_size,
                    grid=torch.zeros(2 * w.grid_size ** 2, dtype=real,
                                     device="cuda"),
                    d_num_skipped=torch.zeros(1, dtype=torch.int64,
                                              device="cuda"),
                    d_norm=torch.zeros(1, dtype=torch.float64, device="cuda"))

    opts = fg.options(accum_mode=accum)
    batch = [job(w, c) for w, c in zip(wls, cubes)]
    fg.grid_batch_device(ws, batch, opts=opts)
    solo = [job(w, c) for w, c in zip(wls, cubes)]
    for j in solo:
        fg.grid_device(ws, j["cube"], j["uu"], j["vv"], j["ww"], j["vis"],
                       j["weight"], j["cell_size_rad"], j["w_scale"],
                       j["grid_size"], j["grid"], j["d_num_skipped"],
                       j["d_norm"], opts=opts)
    torch.cuda.synchronize()
    assert ws.stats().status == 0
    tol_grid = 1e-5 if single else 1e-12
    for w, b, s in zip(wls, batch, solo):
        sk, nrm, g = _oracle(oracle, w, single)
        gb = b["grid"].cpu().numpy()
        gs = s["grid"].cpu().numpy()
        assert int(b["d_num_skipped"].item()) == sk == int(s["d_num_skipped"].item())
        if w.num_points == 0:
            assert not gb.any() and b["d_norm"].item() == 0.0
            continue
        assert rel_rms(gb, g) <= tol_grid
        assert rel_rms(gb, gs) <= (2e-6 if single else 1e-13)
        assert abs(b["d_norm"].item() - nrm) <= 1e-12 * abs(nrm)
        assert b["d_norm"].item() == s["d_norm"].item()
    for c in cubes:
        c.close()
    ws.close()


def test_batch_can_be_graph_captured(oracle):
    wls = _jobs(True)[:3]
    ws = fg.Workspace(0)
    cubes = [fg.Cube(ws, w.support, w.oversample, w.conv_size_half,
                     w.conv_func, data_is_double=False) for w in wls]
    grids = [torch.zeros(2 * w.grid_size ** 2, device="cuda") for w in wls]
    jobs = [dict(cube=c, uu=_dev(w.uu, torch.float32),
                 vv=_dev(w.vv, torch.float32), ww=_dev(w.ww, torch.float32),
                 vis=_dev(w.vis, torch.float32),
                 weight=_dev(w.weight, torch.float32),
                 cell_size_rad=float(np.float32(w.cell_size_rad)),
                 w_scale=float(np.float32(w.w_scale)),
                 grid_size=w.grid_size, grid=g)
            for w, c, g in zip(wls, cubes, grids)]
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        fg.grid_batch_device(ws, jobs, stream=s)   # sizes the buffers
    s.synchronize()
    for g in grids:
        g.zero_()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        fg.grid_batch_device(ws, jobs, stream=s)
    # torch replays a graph on the current stream: make that the stream the
    # workspace's buffers are used on.
    with torch.cuda.stream(s):
        graph.replay()
        graph.replay()
    torch.cuda.synchronize()
    for w, g in zip(wls, grids):
        if w.num_points == 0:
            continue
        _, _, ref = _oracle(oracle, w, True)
        # two replays accumulate twice
        assert rel_rms(g.cpu().numpy(), 2 * ref) <= 1e-5
    del graph
    for c in cubes:
        c.close()
    ws.close()
