"""Uniform weighting on the GPU (utils/oskar_grid_weights.c:38-172)
against the reference's fixtures and the oracle.  Tolerances:
  drop-ins and ordered device write: bit-exact (skip counts, every grid
    cell, every output weight), FP64 and FP32;
  atomic device write: bit-exact for unit weights; otherwise each cell
    within 1e-12 (FP64) / 1e-5 (FP32) relative of the ordered sum, since
    only the order of the additions differs."""
import numpy as np
import pytest
import torch

from conftest import load_weights_golden
import fpga_gridding_b200 as fg
from fpga_gridding_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ws():
    w = fg.Workspace(0)
    yield w
    w.close()


@pytest.mark.parametrize("name", ["weights_d", "weights_f"])
def test_dropin_weights_match_reference_fixture(name):
    z = load_weights_golden(name)
    single = bool(z["single"])
    write = fg.oskar_grid_weights_write_f if single else \
        fg.oskar_grid_weights_write_d
    read = fg.oskar_grid_weights_read_f if single else \
        fg.oskar_grid_weights_read_d
    g = int(z["grid_size"])
    grid = z["grid"].copy()
    wout = z["weight_out"].copy()
    n = z["uu"].size
    sk_w = write(n, z["uu"], z["vv"], z["weight"], z["cell_size_rad"], g,
                 grid)
    sk_r = read(n, z["uu"], z["vv"], z["weight"], wout, z["cell_size_rad"],
                g, grid)
    assert sk_w == int(z["out_skipped_write"])
    assert sk_r == int(z["out_skipped_read"])
    assert np.array_equal(grid, z["out_grid"])
    assert np.array_equal(wout, z["out_weight"])


def _uv_case(seed=4):
    """plain_small's uv points at twice the cell size (the longest
    baselines then fall outside the grid) plus 64 points far outside."""
    w = W.plain_small().numpy()
    rng = np.random.default_rng(seed)
    far = rng.choice([-1.0, 1.0], (2, 64)) * 1e3 * np.abs(w["uu"]).max()
    uu = np.concatenate([w["uu"], far[0]])
    vv = np.concatenate([w["vv"], far[1]])
    n = uu.size
    return dict(uu=uu, vv=vv, weight=rng.uniform(0.1, 2.0, n),
                cell=w["cell_size_rad"] * 2.0, g=w["grid_size"],
                grid=rng.uniform(0.0, 1.0, w["grid_size"] ** 2),
                wout=rng.uniform(-1.0, 1.0, n))


@pytest.mark.parametrize("single", [False, True])
def test_device_ordered_write_and_read_bit_exact(ws, oracle, single):
    c = _uv_case()
    real = np.float32 if single else np.float64
    tdt = torch.float32 if single else torch.float64
    sk_w, g_ref, sk_r, w_ref = oracle.weights(
        c["uu"], c["vv"], c["weight"], c["cell"], c["g"], c["grid"],
        c["wout"], single=single)
    assert 64 <= sk_w < c["uu"].size
    cell = float(real(c["cell"]))
    t = {k: torch.as_tensor(np.asarray(c[k], real)).cuda()
         for k in ("uu", "vv", "weight", "grid", "wout")}
    skip = torch.full((1,), 12345, dtype=torch.int64, device="cuda")
    fg.weights_write_device(ws, t["uu"], t["vv"], t["weight"], cell, c["g"],
                            t["grid"], skip)
    torch.cuda.synchronize()
    assert int(skip.item()) == sk_w
    assert np.array_equal(t["grid"].cpu().numpy(), g_ref)
    fg.weights_read_device(ws, t["uu"], t["vv"], t["weight"], t["wout"],
                           cell, c["g"], t["grid"], skip)
    torch.cuda.synchronize()
    assert int(skip.item()) == sk_r
    assert np.array_equal(t["wout"].cpu().numpy(), w_ref)
    assert t["wout"].dtype == tdt


@pytest.mark.parametrize("single", [False, True])
def test_device_atomic_write_within_tolerance(ws, oracle, single):
    c = _uv_case(seed=9)
    real = np.float32 if single else np.float64
    cell = float(real(c["cell"]))
    zero = np.zeros(c["g"] ** 2)
    sk_w, g_ref, _, _ = oracle.weights(c["uu"], c["vv"], c["weight"],
                                       c["cell"], c["g"], zero, c["wout"],
                                       single=single)
    t = {k: torch.as_tensor(np.asarray(c[k], real)).cuda()
         for k in ("uu", "vv", "weight")}
    grid = torch.zeros(c["g"] ** 2, dtype=t["uu"].dtype, device="cuda")
    skip = torch.zeros(1, dtype=torch.int64, device="cuda")
    fg.weights_write_device(ws, t["uu"], t["vv"], t["weight"], cell, c["g"],
                            grid, skip, ordered=False)
    torch.cuda.synchronize()
    assert int(skip.item()) == sk_w
    got = grid.cpu().numpy().astype(np.float64)
    ref = g_ref.astype(np.float64)
    tol = 1e-5 if single else 1e-12
    nz = ref != 0
    assert np.array_equal(got[~nz], ref[~nz])
    assert np.max(np.abs(got[nz] - ref[nz]) / ref[nz]) <= tol
    # Unit weights: every partial sum is an exact integer.
    grid.zero_()
    ones = torch.ones_like(t["uu"])
    fg.weights_write_device(ws, t["uu"], t["vv"], ones, cell, c["g"], grid,
                            skip, ordered=False)
    _, g1, _, _ = oracle.weights(c["uu"], c["vv"], np.ones(c["uu"].size),
                                 c["cell"], c["g"], zero, c["wout"],
                                 single=single)
    torch.cuda.synchronize()
    assert np.array_equal(grid.cpu().numpy(), g1)


def test_empty_and_all_skipped(ws):
    g = 32
    grid = torch.rand(g * g, dtype=torch.float64, device="cuda")
    before = grid.clone()
    skip = torch.full((1,), 7, dtype=torch.int64, device="cuda")
    e = torch.empty(0, dtype=torch.float64, device="cuda")
    fg.weights_write_device(ws, e, e, e, 1.0 / g, g, grid, skip)
    torch.cuda.synchronize()
    assert int(skip.item()) == 0 and torch.equal(grid, before)
    far = torch.full((100,), 1e6, dtype=torch.float64, device="cuda")
    w = torch.ones(100, dtype=torch.float64, device="cuda")
    out = torch.full((100,), 3.0, dtype=torch.float64, device="cuda")
    for ordered in (True, False):
        fg.weights_write_device(ws, far, far, w, 1.0 / g, g, grid, skip,
                                ordered=ordered)
        torch.cuda.synchronize()
        assert int(skip.item()) == 100 and torch.equal(grid, before)
    fg.weights_read_device(ws, far, far, w, out, 1.0 / g, g, grid, skip)
    torch.cuda.synchronize()
    assert int(skip.item()) == 100
    assert torch.all(out == 3.0)


def test_full_size_unit_weight_properties(ws):
    """8192^2 weights grid, 20 M points: with unit weights the ordered and
    atomic writes agree exactly, the grid sums to the kept points, and
    read gives 1 / count at every kept point."""
    g = 8192
    n = 20_000_000
    gen = torch.Generator(device="cuda").manual_seed(3)
    uu = torch.randn(n, generator=gen, device="cuda") * 1500.0
    vv = torch.randn(n, generator=gen, device="cuda") * 1500.0
    cell = 1.0 / 4096.0
    ones = torch.ones(n, device="cuda")
    a = torch.zeros(g * g, device="cuda")
    b = torch.zeros(g * g, device="cuda")
    sa = torch.zeros(1, dtype=torch.int64, device="cuda")
    sb = torch.zeros(1, dtype=torch.int64, device="cuda")
    fg.weights_write_device(ws, uu, vv, ones, cell, g, a, sa, ordered=True)
    fg.weights_write_device(ws, uu, vv, ones, cell, g, b, sb, ordered=False)
    torch.cuda.synchronize()
    assert int(sa.item()) == int(sb.item())
    assert torch.equal(a, b)
    kept = n - int(sa.item())
    assert 0 < kept < n
    assert float(a.double().sum().item()) == float(kept)
    out = torch.zeros(n, device="cuda")
    fg.weights_read_device(ws, uu, vv, ones, out, cell, g, a, sa)
    torch.cuda.synchronize()
    assert int(sa.item()) == n - kept
    # every kept point's weight is 1 / (its cell's count): they sum to the
    # number of occupied cells
    occupied = int((a > 0).sum().item())
    assert abs(float(out.double().sum().item()) - occupied) <= 1e-3 * occupied


@pytest.mark.parametrize("single", [False, True])
def test_ordered_write_run_lengths_bit_exact(ws, oracle, single):
    """Cells holding 1, 31, 32, 33, 63, 64, 65, 1000 and 3811 points in
    shuffled order with non-integer weights: runs handled by one thread,
    by a warp, ending exactly on a 32-point chunk and spanning many."""
    g = 16
    rng = np.random.default_rng(17)
    counts = [1, 31, 32, 33, 63, 64, 65, 1000, 3811]
    cells = rng.choice(g * g, size=len(counts), replace=False)
    pts = np.concatenate([np.full(c, cell) for c, cell in zip(counts, cells)])
    rng.shuffle(pts)
    gu = pts % g - g // 2
    gv = pts // g - g // 2
    # grid_scale = 1: positions in cells, jittered inside the cell
    uu = -(gu + rng.uniform(-0.4, 0.4, pts.size))
    vv = gv + rng.uniform(-0.4, 0.4, pts.size)
    wt = rng.uniform(0.01, 10.0, pts.size)
    grid0 = rng.uniform(0.0, 1.0, g * g)
    real = np.float32 if single else np.float64
    sk, g_ref, _, _ = oracle.weights(uu, vv, wt, 1.0 / g, g, grid0,
                                     np.zeros(pts.size), single=single)
    assert sk == 0
    t = {k: torch.as_tensor(np.asarray(a, real)).cuda()
         for k, a in (("uu", uu), ("vv", vv), ("w", wt), ("grid", grid0))}
    fg.weights_write_device(ws, t["uu"], t["vv"], t["w"], 1.0 / g, g,
                            t["grid"])
    torch.cuda.synchronize()
    assert np.array_equal(t["grid"].cpu().numpy(), g_ref)
