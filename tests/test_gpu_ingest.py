"""Ingest on the GPU: coordinates in metres scaled to wavelengths inside the
prep and weighting kernels exactly as scale_coords (utils/read_vis.c:51-73)
does on the host, and host visibility blocks streamed through
oskar_b200_blocks_* as the reference's main loop reads them
(main.cpp:413-535).  The comparison is the CPU pipeline: scale_coords, then
the oracle.  Tolerances: skip counts and weights bit-exact; grid relative
RMS 1e-12 (FP64) / 1e-5 (FP32, vs the FP64 oracle on the same float
inputs); norm 1e-12."""
import ctypes as C

import numpy as np
import pytest
import torch

import fpga_gridding_b200 as fg
from fpga_gridding_b200 import _lib, workloads as W

pytestmark = pytest.mark.gpu

FREQ = 149.7e6
C_LIGHT = 299792458.0


@pytest.fixture(scope="module")
def ws():
    w = fg.Workspace(0)
    yield w
    w.close()


def _metres_job(single):
    """plain_small with its coordinates expressed in metres at FREQ."""
    w = W.plain_small().numpy()
    real = np.float32 if single else np.float64
    m = {k: np.asarray(w[k] * (C_LIGHT / FREQ), real)
         for k in ("uu", "vv", "ww")}
    return w, m, real


def _cpu_pipeline(oracle, w, m, real, single):
    """scale_coords on the host, then the FP64 oracle (on the float values
    for FP32)."""
    su, sv, sw = oracle.scale_coords(FREQ, m["uu"], m["vv"], m["ww"])
    ref = dict(w)
    for k, a in (("uu", su), ("vv", sv), ("ww", sw)):
        ref[k] = np.asarray(a, np.float64)
    if single:
        for k in ("conv_func", "vis", "weight"):
            ref[k] = np.asarray(w[k], np.float32).astype(np.float64)
        ref["cell_size_rad"] = float(np.float32(w["cell_size_rad"]))
        ref["w_scale"] = float(np.float32(w["w_scale"]))
    return oracle.grid_d(ref, threads=8), ref


def _scalars(w, single):
    if single:
        return float(np.float32(w["cell_size_rad"])), \
            float(np.float32(w["w_scale"]))
    return w["cell_size_rad"], w["w_scale"]


@pytest.mark.parametrize("single", [False, True])
def test_grid_with_frequency_matches_scale_then_grid(ws, oracle, single):
    w, m, real = _metres_job(single)
    (s1, n1, g1), _ = _cpu_pipeline(oracle, w, m, real, single)
    cube = fg.Cube(ws, w["support"], w["oversample"], w["conv_size_half"],
                   np.asarray(w["conv_func"], real), data_is_double=not single)
    g = w["grid_size"]
    tdt = torch.float32 if single else torch.float64
    grid = torch.zeros(2 * g * g, dtype=tdt, device="cuda")
    skip = torch.zeros(1, dtype=torch.int64, device="cuda")
    norm = torch.zeros(1, dtype=torch.float64, device="cuda")
    cell, wsc = _scalars(w, single)
    d = lambda a: torch.as_tensor(np.asarray(a, real)).cuda()
    fg.grid_device(ws, cube, d(m["uu"]), d(m["vv"]), d(m["ww"]), d(w["vis"]),
                   d(w["weight"]), cell, wsc, g, grid, skip, norm,
                   opts=fg.options(frequency_hz=FREQ))
    torch.cuda.synchronize()
    assert int(skip.item()) == s1
    tol = 1e-5 if single else 1e-12
    assert oracle.rel_rms(grid.cpu().numpy(), g1) <= tol
    assert abs(norm.item() - n1) <= 1e-12 * abs(n1)
    cube.close()


@pytest.mark.parametrize("single", [False, True])
def test_blocks_stream_matches_cpu_pipeline(ws, oracle, single):
    """Seven uneven host blocks (one empty) in metres through the block
    ingest: the same grid, norm and skip count as scaling and gridding the
    whole job on the CPU."""
    w, m, real = _metres_job(single)
    (s1, n1, g1), _ = _cpu_pipeline(oracle, w, m, real, single)
    cube = fg.Cube(ws, w["support"], w["oversample"], w["conv_size_half"],
                   np.asarray(w["conv_func"], real), data_is_double=not single)
    g = w["grid_size"]
    tdt = torch.float32 if single else torch.float64
    grid = torch.zeros(2 * g * g, dtype=tdt, device="cuda")
    norm = torch.zeros(1, dtype=torch.float64, device="cuda")
    cell, wsc = _scalars(w, single)
    n = m["uu"].size
    edges = [0, 1000, 1000, 37000, 90001, 150000, 200000, n]
    vis = np.asarray(w["vis"], real)
    blocks = fg.Blocks(ws, cube, cell, wsc, g, grid, norm)
    # The caller's buffers are refilled for every block, as main.cpp does.
    buf = {k: np.empty(max(np.diff(edges)), real) for k in ("uu", "vv", "ww")}
    vbuf = np.empty(2 * max(np.diff(edges)), real)
    for a, b in zip(edges[:-1], edges[1:]):
        k = b - a
        for key in buf:
            buf[key][:k] = m[key][a:b]
        vbuf[:2 * k] = vis[2 * a:2 * b]
        blocks.push(buf["uu"][:k], buf["vv"][:k], buf["ww"][:k],
                    vbuf[:2 * k], frequency_hz=FREQ)
        for key in buf:
            buf[key][:k] = np.nan   # the copies have landed
        vbuf[:2 * k] = np.nan
    skipped = blocks.finish()
    blocks.close()
    assert skipped == s1
    tol = 1e-5 if single else 1e-12
    assert oracle.rel_rms(grid.cpu().numpy(), g1) <= tol
    assert abs(norm.item() - n1) <= 1e-12 * abs(n1)
    cube.close()


@pytest.mark.parametrize("single", [False, True])
def test_weights_with_frequency_bit_exact(ws, oracle, single):
    w, m, real = _metres_job(single)
    su, sv, _ = oracle.scale_coords(FREQ, m["uu"], m["vv"], m["ww"])
    g = w["grid_size"]
    cell = float(real(w["cell_size_rad"]))
    rng = np.random.default_rng(3)
    wt = rng.uniform(0.1, 2.0, su.size)
    sk_w, g_ref, sk_r, w_ref = oracle.weights(
        su, sv, wt, cell, g, np.zeros(g * g), np.zeros(su.size),
        single=single)
    d = lambda a: torch.as_tensor(np.asarray(a, real)).cuda()
    grid = torch.zeros(g * g, dtype=d(su).dtype, device="cuda")
    out = torch.zeros(su.size, dtype=grid.dtype, device="cuda")
    skip = torch.zeros(1, dtype=torch.int64, device="cuda")
    fg.weights_write_device(ws, d(m["uu"]), d(m["vv"]), d(wt), cell, g, grid,
                            skip, frequency_hz=FREQ)
    torch.cuda.synchronize()
    assert int(skip.item()) == sk_w
    assert np.array_equal(grid.cpu().numpy(), g_ref)
    fg.weights_read_device(ws, d(m["uu"]), d(m["vv"]), d(wt), out, cell, g,
                           grid, skip, frequency_hz=FREQ)
    torch.cuda.synchronize()
    assert int(skip.item()) == sk_r
    assert np.array_equal(out.cpu().numpy(), w_ref)


def test_invalid_frequency_rejected(ws):
    w = W.plain_small().numpy()
    cube = fg.Cube(ws, w["support"], w["oversample"], w["conv_size_half"],
                   np.asarray(w["conv_func"], np.float32),
                   data_is_double=False)
    g = w["grid_size"]
    grid = torch.zeros(2 * g * g, device="cuda")
    t = torch.zeros(4, device="cuda")
    vis = torch.zeros(8, device="cuda")
    for f in (-1.0, float("nan"), float("inf")):
        with pytest.raises(fg.GridderError):
            fg.grid_device(ws, cube, t, t, t, vis, t, 1e-5, 1.0, g, grid,
                           opts=fg.options(frequency_hz=f))
    blocks = fg.Blocks(ws, cube, 1e-5, 1.0, g, grid)
    with pytest.raises(fg.GridderError):
        blocks.push(np.zeros(4), np.zeros(4), np.zeros(4), np.zeros(8),
                    frequency_hz=-5.0)
    assert blocks.finish() == 0
    blocks.close()
    cube.close()


@pytest.mark.parametrize("single", [False, True])
@pytest.mark.parametrize("kt", [_lib.KERNEL_NATIVE, _lib.KERNEL_F16])
def test_planar_cube_equals_interleaved(ws, single, kt):
    """The real and imaginary cubes of the two kernel FITS files, given
    separately: the same resident cube as the interleaved one the
    reference's main loop builds (main.cpp:197-201): equal size, the same
    norm to the bit (the norm table reads the real parts), and grids equal
    up to the order of the grid atomics."""
    if single is False and kt != _lib.KERNEL_NATIVE:
        pytest.skip("FP64 data uses native kernels")
    w = W.plain_small().numpy()
    real = np.float32 if single else np.float64
    conv = np.asarray(w["conv_func"], real)
    re, im = conv[0::2].copy(), conv[1::2].copy()
    g = w["grid_size"]
    tdt = torch.float32 if single else torch.float64
    d = lambda a: torch.as_tensor(np.asarray(a, real)).cuda()
    cell, wsc = _scalars(w, single)
    outs = []
    for planar in (False, True):
        if planar:
            cube = fg.Cube(ws, w["support"], w["oversample"],
                           w["conv_size_half"], re, data_is_double=not single,
                           kernel_type=kt, conv_imag=im)
        else:
            cube = fg.Cube(ws, w["support"], w["oversample"],
                           w["conv_size_half"], conv,
                           data_is_double=not single, kernel_type=kt)
        grid = torch.zeros(2 * g * g, dtype=tdt, device="cuda")
        norm = torch.zeros(1, dtype=torch.float64, device="cuda")
        fg.grid_device(ws, cube, d(w["uu"]), d(w["vv"]), d(w["ww"]),
                       d(w["vis"]), d(w["weight"]), cell, wsc, g, grid, None,
                       norm)
        torch.cuda.synchronize()
        outs.append((grid.cpu().numpy(), norm.item(), cube.bytes))
        cube.close()
    assert outs[0][1] == outs[1][1] and outs[0][2] == outs[1][2]
    from oracle.oracle import rel_rms
    assert rel_rms(outs[1][0], outs[0][0]) <= (1e-6 if single else 1e-14)
