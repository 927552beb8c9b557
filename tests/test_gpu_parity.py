"""GPU gridder against the CPU oracle (itself pinned bit-exact to the
reference).  Tolerances:
  FP64 drop-in:  grid relative RMS <= 1e-12, norm relative error <= 1e-12
  FP32 drop-in:  grid relative RMS <= 1e-5 against the FP64 oracle on the
                 same (float) inputs, norm relative error <= 1e-12
  placement:     num_skipped and every (cell, plane, offsets, conj)
                 bit-exact, in FP64 and in the reference's float arithmetic.
The relative RMS is the reference harness's metric (main.cpp:575-598)."""
import numpy as np
import pytest
import torch

from conftest import golden_names, load_golden
import fpga_gridding_b200 as fg
from fpga_gridding_b200 import _lib, workloads as W

pytestmark = pytest.mark.gpu

TOL_D = 1e-12
TOL_F = 1e-5


def promote(w):
    """The same inputs as float32 values held in float64 (what the FP64
    oracle sees for an FP32 job)."""
    out = dict(w)
    for k in ("conv_func", "uu", "vv", "ww", "vis", "weight"):
        out[k] = np.asarray(w[k], np.float32).astype(np.float64)
    out["cell_size_rad"] = float(np.float32(w["cell_size_rad"]))
    out["w_scale"] = float(np.float32(w["w_scale"]))
    return out


@pytest.fixture(scope="module")
def small():
    return W.plain_small().numpy()


@pytest.fixture(scope="module")
def ws():
    w = fg.Workspace(0)
    yield w
    w.close()


def dev(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=dtype)).cuda()


# ---------------------------------------------------------------------------
# Drop-in entry points
# ---------------------------------------------------------------------------

def test_dropin_d_matches_oracle(oracle, small):
    s1, n1, g1 = oracle.grid_d(small, threads=8)
    s2, n2, g2 = fg.grid_workload(small, single=False)
    assert s2 == s1
    assert oracle.rel_rms(g2, g1) <= TOL_D
    assert abs(n2 - n1) <= TOL_D * abs(n1)


def test_dropin_f_matches_fp64_oracle(oracle, small):
    s1, n1, g1 = oracle.grid_d(promote(small), threads=8)
    s2, n2, g2 = fg.grid_workload(small, single=True)
    assert s2 == s1
    assert oracle.rel_rms(g2, g1) <= TOL_F
    assert abs(n2 - n1) <= TOL_D * abs(n1)


def test_dropin_accumulates_into_grid_and_norm(oracle, small):
    g = small["grid_size"]
    rng = np.random.default_rng(5)
    base = rng.normal(size=2 * g * g)
    s1, n1, g1 = oracle.grid_d(small, grid_arr=base.copy(), norm=3.5,
                               threads=8)
    s2, n2, g2 = fg.grid_workload(small, single=False, grid=base.copy(),
                                  norm=3.5)
    assert s1 == s2
    assert oracle.rel_rms(g2, g1) <= TOL_D
    assert abs(n2 - n1) <= TOL_D * abs(n1)


def _many_points(n, seed=12):
    """n random visibilities on a 512^2 grid with supports 1 -> 3: enough
    points that the drop-in uploads and grids them in several chunks."""
    rng = np.random.default_rng(seed)
    g, os_ = 512, 4
    support = W.support_ramp(8, 1, 3)
    csh = W.min_conv_size_half(support, os_) + 1
    cube = W.analytic_kernel_cube(support, os_, csh).numpy()
    pos = rng.uniform(-240.0, 240.0, (2, n))
    return dict(num_w_planes=8, support=support, oversample=os_,
                conv_size_half=csh, conv_func=cube, uu=-pos[0] / g,
                vv=pos[1] / g, ww=rng.uniform(-49.0, 49.0, n),
                vis=rng.normal(size=2 * n), weight=np.ones(n),
                cell_size_rad=1.0, w_scale=1.0, grid_size=g)


@pytest.mark.parametrize("single", [False, True])
def test_dropin_pipelined_chunks(oracle, single):
    """5.6 M points: the drop-in uploads them in chunks that are gridded
    while the next chunk and the caller's grid cross PCIe; the result
    matches the oracle as one call does."""
    w = _many_points(5_600_000)
    g = w["grid_size"]
    rng = np.random.default_rng(2)
    real = np.float32 if single else np.float64
    base = rng.normal(size=2 * g * g).astype(real)
    ref_in = promote(w) if single else w
    s1, n1, g1 = oracle.grid_d(ref_in, grid_arr=base.astype(np.float64),
                               norm=1.25, threads=8)
    s2, n2, g2 = fg.grid_workload(w, single=single, grid=base.copy(),
                                  norm=1.25)
    assert s1 == s2
    assert oracle.rel_rms(g2, g1) <= (TOL_F if single else TOL_D)
    # norm is a sum of 5.6 M positive FP64 terms: the reference adds them
    # one by one, the GPU in per-block partials; the two orders may differ
    # by up to n * 2^-53 relative.
    assert abs(n2 - n1) <= max(TOL_D, w["uu"].size * 2.0 ** -53) * abs(n1)


@pytest.mark.parametrize("single", [False, True])
def test_dropin_leaves_cells_no_footprint_reaches_bit_for_bit(oracle,
                                                              single):
    """Two clusters of points on a 512^2 grid.  Rows far from both hold
    NaN and -0.0 in the caller's grid: they come back bit for bit, as the
    reference never touches them (adding a zero contribution would turn
    -0.0 into +0.0); the rest matches the oracle."""
    rng = np.random.default_rng(31)
    g, os_, n = 512, 4, 4000
    support = W.support_ramp(8, 1, 3)
    csh = W.min_conv_size_half(support, os_) + 1
    cube = W.analytic_kernel_cube(support, os_, csh).numpy()
    centre = np.where(np.arange(n) < n // 2, -156.0, 124.0)
    pu = centre + rng.uniform(-20.0, 20.0, n)
    pv = centre + rng.uniform(-20.0, 20.0, n)
    w = dict(num_w_planes=8, support=support, oversample=os_,
             conv_size_half=csh, conv_func=cube, uu=-pu / g, vv=pv / g,
             ww=rng.uniform(-49.0, 49.0, n), vis=rng.normal(size=2 * n),
             weight=np.ones(n), cell_size_rad=1.0, w_scale=1.0, grid_size=g)
    real = np.float32 if single else np.float64
    base = rng.normal(size=(g, g, 2)).astype(real)
    base[250:262, :, 0] = np.nan
    base[250:262, :, 1] = -0.0
    base = base.reshape(-1)
    special = np.zeros((g, g, 2), bool)
    special[250:262] = True
    special = special.reshape(-1)
    ref_in = promote(w) if single else w
    s1, n1, g1 = oracle.grid_d(ref_in, grid_arr=base.astype(np.float64),
                               norm=0.0, threads=8)
    s2, n2, g2 = fg.grid_workload(w, single=single, grid=base.copy(),
                                  norm=0.0)
    assert s1 == s2 == 0
    assert np.array_equal(g2[special].view(np.uint8),
                          base[special].view(np.uint8))
    assert oracle.rel_rms(g2[~special], g1[~special]) <= \
        (TOL_F if single else TOL_D)
    assert abs(n2 - n1) <= TOL_D * abs(n1)


@pytest.mark.parametrize("single", [False, True])
def test_dropin_bands_wider_than_band_height(oracle, single):
    """Supports up to 70 on a 256^2 grid (bands of 64 rows): footprints
    reach past the neighbouring band, so a band's rows go back to the host
    only after the band two further on is gridded.  The drop-in still
    matches the oracle, accumulating into the caller's grid."""
    rng = np.random.default_rng(21)
    g, os_, n = 256, 4, 6000
    support = W.support_ramp(8, 8, 70)
    csh = W.min_conv_size_half(support, os_) + 1
    cube = W.analytic_kernel_cube(support, os_, csh).numpy()
    pos = rng.uniform(-60.0, 60.0, (2, n))
    w = dict(num_w_planes=8, support=support, oversample=os_,
             conv_size_half=csh, conv_func=cube, uu=-pos[0] / g,
             vv=pos[1] / g, ww=rng.uniform(-49.0, 49.0, n),
             vis=rng.normal(size=2 * n), weight=np.ones(n),
             cell_size_rad=1.0, w_scale=1.0, grid_size=g)
    real = np.float32 if single else np.float64
    base = rng.normal(size=2 * g * g).astype(real)
    ref_in = promote(w) if single else w
    s1, n1, g1 = oracle.grid_d(ref_in, grid_arr=base.astype(np.float64),
                               norm=0.5, threads=8)
    s2, n2, g2 = fg.grid_workload(w, single=single, grid=base.copy(),
                                  norm=0.5)
    assert 0 < s1 < n and s1 == s2
    assert oracle.rel_rms(g2, g1) <= (TOL_F if single else TOL_D)
    assert abs(n2 - n1) <= TOL_D * abs(n1)


@pytest.mark.parametrize("name", golden_names())
def test_golden_fixtures(name):
    inputs, out = load_golden(name)
    if out["single"]:
        # The FP32 fixture comes from the reference's float arithmetic:
        # grid it with the same coordinate mode through the extended API.
        ws = fg.Workspace(0)
        cube = fg.Cube(ws, inputs["support"], inputs["oversample"],
                       inputs["conv_size_half"], inputs["conv_func"],
                       data_is_double=False)
        g = inputs["grid_size"]
        grid = torch.zeros(2 * g * g, dtype=torch.float32, device="cuda")
        skip = torch.zeros(1, dtype=torch.int64, device="cuda")
        norm = torch.zeros(1, dtype=torch.float64, device="cuda")
        fg.grid_device(ws, cube, *[dev(inputs[k], np.float32) for k in
                                   ("uu", "vv", "ww", "vis", "weight")],
                       inputs["cell_size_rad"], inputs["w_scale"], g, grid,
                       skip, norm,
                       opts=fg.options(coord_mode=_lib.COORDS_REFERENCE_F32))
        torch.cuda.synchronize()
        assert int(skip.item()) == out["skipped"]
        from oracle.oracle import rel_rms
        assert rel_rms(grid.cpu().numpy(), out["grid"]) <= TOL_F
        assert abs(norm.item() - out["norm"]) <= TOL_D * abs(out["norm"])
        cube.close()
        ws.close()
    else:
        from oracle.oracle import rel_rms
        s, n, grid = fg.grid_workload(inputs, single=False)
        assert s == out["skipped"]
        assert rel_rms(grid, out["grid"]) <= TOL_D
        assert abs(n - out["norm"]) <= TOL_D * max(1.0, abs(out["norm"]))


def test_known_answer_all_ones_exact():
    """All-ones kernel and visibilities: every cell holds an integer hit
    count, exactly representable, so the FP64 result is bit-exact."""
    inputs, out = load_golden("ones_d")
    s, n, grid = fg.grid_workload(inputs, single=False)
    assert s == out["skipped"] and n == out["norm"]
    assert np.array_equal(grid, out["grid"])


def test_empty_input_leaves_grid_and_norm(small):
    w = dict(small)
    for k in ("uu", "vv", "ww", "weight"):
        w[k] = small[k][:0]
    w["vis"] = small["vis"][:0]
    g = w["grid_size"]
    base = np.arange(2 * g * g, dtype=np.float64)
    s, n, grid = fg.grid_workload(w, single=False, grid=base.copy(), norm=2.0)
    assert s == 0 and n == 2.0
    assert np.array_equal(grid, base)


def test_all_points_skipped(small):
    w = dict(small)
    w["uu"] = np.full_like(small["uu"], 1e6)
    s, n, grid = fg.grid_workload(w, single=False, norm=1.25)
    assert s == len(w["uu"]) and n == 1.25
    assert not grid.any()


# ---------------------------------------------------------------------------
# Placement: bit-exact
# ---------------------------------------------------------------------------

def scalars(w, single):
    """cell_size_rad and w_scale as the FP32 drop-in receives them."""
    if single:
        return float(np.float32(w["cell_size_rad"])), float(np.float32(w["w_scale"]))
    return w["cell_size_rad"], w["w_scale"]


def _check_place(ws, oracle, w, single, coord_mode):
    real = np.float32 if single else np.float64
    cell, wsc = scalars(w, single)
    got = fg.place_device(ws, w["support"], w["oversample"],
                          dev(w["uu"], real), dev(w["vv"], real),
                          dev(w["ww"], real), cell, wsc, w["grid_size"],
                          coord_mode=coord_mode)
    got = {k: v.cpu().numpy() for k, v in got.items()}
    if single and coord_mode == _lib.COORDS_F64:
        ref = oracle.place(promote(w))
    else:
        ref = oracle.place(w, single=single)
    assert np.array_equal(got["skipped"], ref["skipped"].astype(np.int32))
    keep = ref["skipped"] == 0
    for k in ("gu", "gv", "plane", "off_u", "off_v", "conj"):
        assert np.array_equal(got[k][keep], ref[k][keep].astype(np.int32)), k


@pytest.mark.parametrize("name", ["edges_d", "odd_oversample_d",
                                  "synth_small_d"])
def test_placement_bit_exact_fp64(ws, oracle, name):
    inputs, _ = load_golden(name)
    _check_place(ws, oracle, inputs, False, _lib.COORDS_F64)
    _check_place(ws, oracle, inputs, True, _lib.COORDS_F64)
    _check_place(ws, oracle, inputs, True, _lib.COORDS_REFERENCE_F32)


def test_placement_bit_exact_small_config(ws, oracle, small):
    _check_place(ws, oracle, small, False, _lib.COORDS_F64)
    _check_place(ws, oracle, small, True, _lib.COORDS_F64)
    _check_place(ws, oracle, small, True, _lib.COORDS_REFERENCE_F32)


# ---------------------------------------------------------------------------
# Launch variants agree
# ---------------------------------------------------------------------------

def _grid_ext(ws, w, single, **opt):
    real = np.float32 if single else np.float64
    tdt = torch.float32 if single else torch.float64
    cube = fg.Cube(ws, w["support"], w["oversample"], w["conv_size_half"],
                   np.asarray(w["conv_func"], real), data_is_double=not single,
                   kernel_type=opt.pop("kernel_type", _lib.KERNEL_NATIVE))
    g = w["grid_size"]
    grid = torch.zeros(2 * g * g, dtype=tdt, device="cuda")
    skip = torch.zeros(1, dtype=torch.int64, device="cuda")
    norm = torch.zeros(1, dtype=torch.float64, device="cuda")
    cell, wsc = scalars(w, single)
    fg.grid_device(ws, cube, *[dev(w[k], real) for k in
                               ("uu", "vv", "ww", "vis", "weight")],
                   cell, wsc, g, grid, skip, norm, opts=fg.options(**opt))
    torch.cuda.synchronize()
    st = ws.stats()
    cube.close()
    return int(skip.item()), float(norm.item()), grid.cpu().numpy(), st


@pytest.mark.parametrize("staging", [1, 2])
@pytest.mark.parametrize("cpt", [1, 2, 4])
def test_launch_variants_fp64(ws, oracle, small, staging, cpt):
    s1, n1, g1 = oracle.grid_d(small, threads=8)
    s2, n2, g2, st = _grid_ext(ws, small, False, staging=staging,
                               classes_per_thread=cpt)
    assert s2 == s1 and st.status == 0
    assert oracle.rel_rms(g2, g1) <= TOL_D
    assert abs(n2 - n1) <= TOL_D * abs(n1)


def _weighted(w, seed=4):
    """The job with weights U(0.25, 4) instead of ones."""
    out = dict(w)
    out["weight"] = np.random.default_rng(seed).uniform(0.25, 4.0,
                                                        len(w["uu"]))
    return out


def test_weighted_gridding_fp64_matches_oracle(ws, oracle, small):
    """apply_weight = 1: each visibility scaled by its weight and the norm
    by tap sum x weight (the reference tiled CUDA gridder's weighting,
    restated in the oracle)."""
    w = _weighted(small)
    s1, n1, g1 = oracle.grid_weighted_d(w)
    s2, n2, g2, st = _grid_ext(ws, w, False, apply_weight=1)
    assert s2 == s1 and st.status == 0
    assert oracle.rel_rms(g2, g1) <= TOL_D
    assert abs(n2 - n1) <= TOL_D * abs(n1)
    # the weights really act: the unweighted grid is far from this one
    _, _, g0 = oracle.grid_d(small, threads=8)
    assert oracle.rel_rms(g0, g1) > 0.1


@pytest.mark.parametrize("staging", [0, 1])
def test_weighted_gridding_fp32_matches_oracle(ws, oracle, small, staging):
    w = _weighted(small)
    s1, n1, g1 = oracle.grid_weighted_d(promote(w))
    s2, n2, g2, st = _grid_ext(ws, w, True, apply_weight=1, staging=staging)
    assert s2 == s1 and st.status == 0
    assert oracle.rel_rms(g2, g1) <= TOL_F
    assert abs(n2 - n1) <= TOL_D * abs(n1)


def test_stats_count_grid_updates(ws, oracle, small):
    _, _, _, st = _grid_ext(ws, small, True)
    assert st.grid_updates == oracle.count_taps(small)
    assert st.num_gridded == len(small["uu"])
    assert st.atomic_flushes == 0  # not counted unless asked for
    # statistics level 3: stage events and the grid atomics counted
    ws._lib.oskar_b200_set_stage_timing(ws.handle, 3)
    try:
        _, _, _, st = _grid_ext(ws, small, True)
    finally:
        ws._lib.oskar_b200_set_stage_timing(ws.handle, 0)
    assert 0 < st.atomic_flushes < st.grid_updates
    assert st.grid_ms > 0


def test_compensated_accumulation(ws, oracle, small):
    """The compensated grid atomics capture the rounding of every grid
    addition: the result is at least as close to the FP64 oracle as the
    plain FP32 one (plain_small piles 241,920 visibilities onto ~80^2
    cells), and within the FP32 bar."""
    _, n1, g1 = oracle.grid_d(promote(small), threads=8)
    _, _, gp, _ = _grid_ext(ws, small, True)
    s, n, gc, st = _grid_ext(ws, small, True,
                             accum_mode=_lib.ACCUM_COMPENSATED)
    ep, ec = oracle.rel_rms(gp, g1), oracle.rel_rms(gc, g1)
    print(f"plain {ep:.3e} compensated {ec:.3e}")
    assert st.status == 0 and s == 0
    assert ec <= TOL_F and ec <= ep
    assert abs(n - n1) <= TOL_D * abs(n1)


def test_compensation_limited_to_the_central_cells(ws, oracle, small):
    """compensate_radius > 0: only tasks whose footprint centre lies within
    that many cells of the grid centre take the compensated flush.  With
    the radius holding about half of the visibilities, the grid lies
    between the plain and the fully compensated ones in accuracy, within
    the FP32 bar, and the norm is unchanged."""
    _, n1, g1 = oracle.grid_d(promote(small), threads=8)
    g = small["grid_size"]
    cell = float(np.float32(small["cell_size_rad"]))
    gu = np.round(-np.asarray(small["uu"], np.float32).astype(np.float64) *
                  float(np.float32(g * cell))) + g // 2
    gv = np.round(np.asarray(small["vv"], np.float32).astype(np.float64) *
                  float(np.float32(g * cell))) + g // 2
    d = np.maximum(np.abs(gu - g // 2), np.abs(gv - g // 2))
    radius = int(np.median(d)) + 1
    _, _, gp, _ = _grid_ext(ws, small, True)
    _, _, gf, _ = _grid_ext(ws, small, True,
                            accum_mode=_lib.ACCUM_COMPENSATED)
    s, n, gr, st = _grid_ext(ws, small, True,
                             accum_mode=_lib.ACCUM_COMPENSATED,
                             compensate_radius=radius)
    ep, ef, er = (oracle.rel_rms(x, g1) for x in (gp, gf, gr))
    print(f"radius {radius}: plain {ep:.3e} central {er:.3e} full {ef:.3e}")
    assert st.status == 0 and s == 0
    assert er <= TOL_F and er <= ep
    assert abs(n - n1) <= TOL_D * abs(n1)


@pytest.mark.parametrize("kt,tol", [(_lib.KERNEL_F16, 2e-3),
                                    (_lib.KERNEL_BF16, 2e-2)])
def test_reduced_precision_kernels(ws, oracle, small, kt, tol):
    s1, n1, g1 = oracle.grid_d(promote(small), threads=8)
    s2, n2, g2, _ = _grid_ext(ws, small, True, kernel_type=kt)
    assert s2 == s1
    err = oracle.rel_rms(g2, g1)
    print(f"kernel_type {kt}: rel RMS vs FP64 oracle {err:.3e}")
    assert err <= tol
    assert abs(n2 - n1) <= TOL_D * abs(n1)
