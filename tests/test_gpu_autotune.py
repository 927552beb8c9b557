"""The autotuner (oskar_b200_autotune): it measures a classes-per-thread
choice for each support size present in the sample, a tile width and
kernel-value path, and with compensated accumulation a compensation radius;
the workspace then grids with those choices, and the result still matches
the oracle (they change the thread layout, the work order and which cells
are compensated, never the arithmetic of a tap).  Tolerance: FP32 grid
relative RMS 1e-5 against the FP64 oracle on the same float inputs."""
import numpy as np
import pytest
import torch

import fpga_gridding_b200 as fg
from fpga_gridding_b200 import workloads as W

pytestmark = pytest.mark.gpu

ALLOWED = {1, 2, 3, 4, 5, 6}


def test_autotune_then_grid_matches_oracle(oracle):
    w = W.plain_small().numpy()
    real = np.float32
    d = lambda a: torch.as_tensor(np.asarray(a, real)).cuda()
    ws = fg.Workspace(0)
    cube = fg.Cube(ws, w["support"], w["oversample"], w["conv_size_half"],
                   np.asarray(w["conv_func"], real), data_is_double=False)
    g = w["grid_size"]
    cell = float(real(w["cell_size_rad"]))
    wsc = float(real(w["w_scale"]))
    model = ws.tune_table()
    scratch = torch.zeros(2 * g * g, device="cuda")
    table = ws.autotune(cube, d(w["uu"]), d(w["vv"]), d(w["ww"]),
                        d(w["vis"]), cell, wsc, g, scratch)
    assert set(table.tolist()) <= ALLOWED
    assert np.array_equal(ws.tune_table(), table)
    ref = dict(w)
    for k in ("conv_func", "uu", "vv", "ww", "vis", "weight"):
        ref[k] = np.asarray(w[k], real).astype(np.float64)
    ref["cell_size_rad"], ref["w_scale"] = cell, wsc
    # supports with too few sample points keep the cost model's choice
    # (placements are bit-exact, so these counts are the device's)
    p = oracle.place(ref)
    kept = p["skipped"] == 0
    counts = np.bincount(np.asarray(w["support"])[p["plane"][kept]],
                         minlength=128)
    for s in range(128):
        if counts[s] < 2000:
            assert table[s] == model[s]
    grid = torch.zeros(2 * g * g, device="cuda")
    fg.grid_device(ws, cube, d(w["uu"]), d(w["vv"]), d(w["ww"]), d(w["vis"]),
                   d(w["weight"]), cell, wsc, g, grid)
    torch.cuda.synchronize()
    _, _, g1 = oracle.grid_d(ref, threads=8)
    assert oracle.rel_rms(grid.cpu().numpy(), g1) <= 1e-5
    cube.close()
    ws.close()


def test_tune_table_set_and_reject():
    ws = fg.Workspace(0)
    t = np.full(128, 3, np.uint8)
    assert np.array_equal(ws.tune_table(t), t)
    bad = t.copy()
    bad[5] = 7
    with pytest.raises(fg.GridderError):
        ws.tune_table(bad)
    assert np.array_equal(ws.tune_table(), t)
    ws.close()


def _f32(w):
    ref = dict(w)
    for k in ("conv_func", "uu", "vv", "ww", "vis", "weight"):
        ref[k] = np.asarray(w[k], np.float32).astype(np.float64)
    ref["cell_size_rad"] = float(np.float32(w["cell_size_rad"]))
    ref["w_scale"] = float(np.float32(w["w_scale"]))
    return ref


def test_autotune_compensated_launch_shape_then_batch_matches_oracle(oracle):
    """Tuned with compensated accumulation: the launch shape is valid (L1
    kernel values, as compensation needs), and a batch of two jobs whose
    options leave tile width, path and radius to the workspace matches the
    FP64 oracle job by job."""
    from fpga_gridding_b200 import _lib
    wa = W.plain_small().numpy()
    wb = W.plain_small(seed=5, num_stations=40, num_times=60, grid_size=512,
                       num_w_planes=12).numpy()
    d = lambda a: torch.as_tensor(np.asarray(a, np.float32)).cuda()
    ws = fg.Workspace(0)
    comp = fg.options(accum_mode=_lib.ACCUM_COMPENSATED)
    cubes = [fg.Cube(ws, w["support"], w["oversample"], w["conv_size_half"],
                     np.asarray(w["conv_func"], np.float32),
                     data_is_double=False) for w in (wa, wb)]
    g = wa["grid_size"]
    scratch = torch.zeros(2 * g * g, device="cuda")
    ws.autotune(cubes[0], d(wa["uu"]), d(wa["vv"]), d(wa["ww"]),
                d(wa["vis"]), float(np.float32(wa["cell_size_rad"])),
                float(np.float32(wa["w_scale"])), g, scratch, opts=comp)
    tile_shift, staging, radius = ws.tune_launch()
    assert tile_shift == 0 or 6 <= tile_shift <= 15
    assert staging == 2 and radius >= 0
    auto = fg.options(accum_mode=_lib.ACCUM_COMPENSATED, compensate_radius=-1)
    jobs = []
    for w, c in zip((wa, wb), cubes):
        gs = w["grid_size"]
        jobs.append(dict(cube=c, uu=d(w["uu"]), vv=d(w["vv"]), ww=d(w["ww"]),
                         vis=d(w["vis"]), weight=d(w["weight"]),
                         cell_size_rad=float(np.float32(w["cell_size_rad"])),
                         w_scale=float(np.float32(w["w_scale"])),
                         grid_size=gs,
                         grid=torch.zeros(2 * gs * gs, device="cuda"),
                         d_num_skipped=torch.zeros(1, dtype=torch.int64,
                                                   device="cuda"),
                         d_norm=torch.zeros(1, dtype=torch.float64,
                                            device="cuda")))
    fg.grid_batch_device(ws, jobs, opts=auto)
    torch.cuda.synchronize()
    for w, j in zip((wa, wb), jobs):
        s, n, ref = oracle.grid_d(_f32(w), threads=8)
        assert int(j["d_num_skipped"].item()) == s
        assert abs(j["d_norm"].item() - n) <= 1e-12 * abs(n)
        assert oracle.rel_rms(j["grid"].cpu().numpy(), ref) <= 1e-5
    for c in cubes:
        c.close()
    ws.close()


def test_tune_launch_set_and_reject():
    ws = fg.Workspace(0)
    assert ws.tune_launch() == (0, 2, 0)
    assert ws.tune_launch((8, 1, 100)) == (8, 1, 100)
    for bad in ((5, 2, 0), (16, 2, 0), (0, 3, 0), (0, 2, -1)):
        with pytest.raises(fg.GridderError):
            ws.tune_launch(bad)
    assert ws.tune_launch() == (8, 1, 100)
    ws.close()
