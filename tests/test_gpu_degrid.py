"""Degridding on the GPU (oskar_b200_degrid): the adjoint of the gridder,
defined in the oracle (orc_degrid_wproj_d) because the reference has none
(Defines.h:48).  Tolerances: skip counts bit-exact and skipped outputs
untouched; FP64 relative RMS over the visibilities 1e-12; FP32 1e-5 against
the FP64 oracle on the same float inputs; the adjoint identity
<grid(v), g> = <v, degrid(g)> to 1e-10 (FP64, 5.6 M visibilities)."""
import numpy as np
import pytest
import torch

from conftest import golden_names, load_golden
import fpga_gridding_b200 as fg
from fpga_gridding_b200 import _lib, workloads as W
from oracle.oracle import rel_rms

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ws():
    w = fg.Workspace(0)
    yield w
    w.close()


def _promote(w):
    out = dict(w)
    for k in ("conv_func", "uu", "vv", "ww", "vis", "weight"):
        out[k] = np.asarray(w[k], np.float32).astype(np.float64)
    out["cell_size_rad"] = float(np.float32(w["cell_size_rad"]))
    out["w_scale"] = float(np.float32(w["w_scale"]))
    return out


def _degrid(ws, w, grid_np, single, kernel_type=_lib.KERNEL_NATIVE,
            fill=7.0, **opt):
    real = np.float32 if single else np.float64
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a, real)).cuda()
    cube = fg.Cube(ws, w["support"], w["oversample"], w["conv_size_half"],
                   np.asarray(w["conv_func"], real), data_is_double=not single,
                   kernel_type=kernel_type)
    n = len(w["uu"])
    vis = torch.full((2 * n,), fill, dtype=d(w["uu"]).dtype, device="cuda")
    skip = torch.zeros(1, dtype=torch.int64, device="cuda")
    cell = float(real(w["cell_size_rad"]))
    wsc = float(real(w["w_scale"]))
    fg.degrid_device(ws, cube, d(w["uu"]), d(w["vv"]), d(w["ww"]),
                     d(w["weight"]), cell, wsc, w["grid_size"], d(grid_np),
                     vis, skip, opts=fg.options(**opt))
    torch.cuda.synchronize()
    cube.close()
    return int(skip.item()), vis.cpu().numpy().astype(np.float64)


def _random_grid(g, seed=5):
    return np.random.default_rng(seed).normal(size=2 * g * g)


def test_degrid_fp64_matches_oracle(ws, oracle):
    w = W.plain_small().numpy()
    gr = _random_grid(w["grid_size"])
    s1, v1 = oracle.degrid_d(w, gr)
    s2, v2 = _degrid(ws, w, gr, False)
    assert s1 == s2
    assert rel_rms(v2, v1) <= 1e-12


def test_degrid_fp32_matches_fp64_oracle(ws, oracle):
    w = W.plain_small().numpy()
    gr = _random_grid(w["grid_size"]).astype(np.float32)
    s1, v1 = oracle.degrid_d(_promote(w), gr.astype(np.float64))
    s2, v2 = _degrid(ws, w, gr, True)
    assert s1 == s2
    assert rel_rms(v2, v1) <= 1e-5


@pytest.mark.parametrize("name", golden_names())
def test_degrid_edge_fixtures(ws, oracle, name):
    """The gridding fixtures' inputs (half-way placements, footprints on and
    past every grid edge, plane clamping, conjugation, far points): skipped
    visibilities keep their value, the others match the oracle."""
    inputs, out = load_golden(name)
    if out["single"]:
        pytest.skip("FP32 fixture uses the reference's float placement")
    gr = _random_grid(inputs["grid_size"], seed=9)
    s1, v1 = oracle.degrid_d(inputs, gr, vis_out=np.full(
        2 * len(inputs["uu"]), 7.0))
    s2, v2 = _degrid(ws, inputs, gr, False, fill=7.0)
    assert s1 == s2 == out["skipped"]
    assert np.array_equal(v1 == 7.0, v2 == 7.0)
    assert rel_rms(v2, v1) <= 1e-12


def test_degrid_is_adjoint_of_grid_at_size(ws):
    """<grid(v), g> = <v, degrid(g)> through the GPU gridder and degridder
    (FP64) on 5.6 M visibilities with a random grid."""
    rng = np.random.default_rng(12)
    n, g, os_ = 5_600_000, 512, 4
    support = W.support_ramp(8, 1, 3)
    csh = W.min_conv_size_half(support, os_) + 1
    cube_np = W.analytic_kernel_cube(support, os_, csh).numpy()
    pos = rng.uniform(-240.0, 240.0, (2, n))
    d = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float64)).cuda()
    uu, vv = d(-pos[0] / g), d(pos[1] / g)
    ww = d(rng.uniform(-49.0, 49.0, n))
    vis = d(rng.normal(size=2 * n))
    wt = d(np.ones(n))
    cube = fg.Cube(ws, support, os_, csh, cube_np, data_is_double=True)
    grid = torch.zeros(2 * g * g, dtype=torch.float64, device="cuda")
    fg.grid_device(ws, cube, uu, vv, ww, vis, wt, 1.0, 1.0, g, grid)
    gr = d(rng.normal(size=2 * g * g))
    out = torch.zeros_like(vis)
    fg.degrid_device(ws, cube, uu, vv, ww, wt, 1.0, 1.0, g, gr, out)
    torch.cuda.synchronize()
    c = lambda t: torch.complex(t[0::2], t[1::2])
    lhs = torch.vdot(c(gr), c(grid)).item()
    rhs = torch.vdot(c(out), c(vis)).item()
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)
    cube.close()


def test_degrid_weights_and_reduced_precision(ws, oracle):
    w = W.plain_small().numpy()
    rng = np.random.default_rng(4)
    w = dict(w)
    w["weight"] = rng.uniform(0.5, 2.0, len(w["uu"]))
    gr = _random_grid(w["grid_size"])
    s1, v1 = oracle.degrid_d(w, gr)
    s2, v2 = _degrid(ws, w, gr, False, apply_weight=1)
    ref = v1.copy()
    ref[0::2] *= w["weight"]
    ref[1::2] *= w["weight"]
    assert rel_rms(v2, ref) <= 1e-12
    s3, v3 = oracle.degrid_d(_promote(w), gr.astype(np.float32).astype(
        np.float64))
    for kt, tol in ((_lib.KERNEL_F16, 2e-3), (_lib.KERNEL_BF16, 1e-2)):
        s4, v4 = _degrid(ws, w, gr.astype(np.float32), True, kernel_type=kt)
        assert s4 == s3
        err = rel_rms(v4, v3)
        print(f"kernel_type {kt}: degrid rel RMS vs FP64 oracle {err:.3e}")
        assert err <= tol


@pytest.mark.parametrize("single", [True, False])
def test_degrid_host_matches_device_call(ws, single):
    """oskar_b200_degrid_host (host arrays, 5.6 M visibilities uploaded in
    chunks that are degridded as they land) gives the device call's values
    bit for bit, the same skip count, and leaves skipped entries of `vis`
    as the caller had them."""
    rng = np.random.default_rng(13)
    real = np.float32 if single else np.float64
    n, g, os_ = 5_600_000, 512, 4
    support = W.support_ramp(8, 1, 3)
    csh = W.min_conv_size_half(support, os_) + 1
    cube_np = W.analytic_kernel_cube(support, os_, csh).numpy().astype(real)
    # a few points fall off the grid edge (skipped)
    pos = rng.uniform(-258.0, 258.0, (2, n))
    h = dict(uu=(-pos[0] / g).astype(real), vv=(pos[1] / g).astype(real),
             ww=rng.uniform(-49.0, 49.0, n).astype(real))
    grid = rng.normal(size=2 * g * g).astype(real)
    cube = fg.Cube(ws, support, os_, csh, cube_np, data_is_double=not single)
    vis_host = np.full(2 * n, 3.5, dtype=real)
    skipped = fg.degrid_host(ws, cube, h["uu"], h["vv"], h["ww"], None, 1.0,
                             1.0, g, grid, vis_host)
    d = lambda a: torch.as_tensor(a).cuda()
    vis_dev = torch.full((2 * n,), 3.5, dtype=d(h["uu"]).dtype, device="cuda")
    skip = torch.zeros(1, dtype=torch.int64, device="cuda")
    fg.degrid_device(ws, cube, d(h["uu"]), d(h["vv"]), d(h["ww"]), None,
                     1.0, 1.0, g, d(grid), vis_dev, skip)
    torch.cuda.synchronize()
    cube.close()
    assert 0 < skipped < n and skipped == int(skip.item())
    assert np.array_equal(vis_host, vis_dev.cpu().numpy())
    assert np.count_nonzero(vis_host == 3.5) >= 2 * skipped
