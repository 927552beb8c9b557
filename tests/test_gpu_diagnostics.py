"""GPU parity of oskar_grid_wproj_f_diagnostics (oskar_grid_wproj.c:245-370)
through the C ABI: the float-coordinate FP32 gridding plus the per-support,
per-plane and per-cell hit counts, against the reference's own outputs
(golden fixture) and the oracle restatement.  Counts and per-cell sums are
exact; the grid is within the FP32 tolerance of the other parity tests."""
import numpy as np
import pytest

import fpga_gridding_b200 as fg
from conftest import load_diag_golden
from fpga_gridding_b200 import _lib, workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_F = 1e-5    # relative RMS of FP32 grids against the reference / oracle


def rel_rms(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) /
                 max(np.sqrt(np.mean(b ** 2)), 1e-300))


def run_gpu(w, init, copy=True):
    """The drop-in on `init` (on copies of it unless copy is False);
    returns the outputs as a dict."""
    o = {k: (v if k == "norm" or not copy else np.array(v, copy=True))
         for k, v in init.items()}
    f32 = lambda k: np.ascontiguousarray(w[k], dtype=np.float32)
    sk, nrm = fg.oskar_grid_wproj_f_diagnostics(
        w["num_w_planes"], w["support"], w["oversample"], w["conv_size_half"],
        f32("conv_func"), len(w["uu"]), f32("uu"), f32("vv"), f32("ww"),
        f32("vis"), f32("weight"), w["cell_size_rad"], w["w_scale"],
        w["grid_size"], o["norm"], o["grid"], o["num_vis_per_wsupport"],
        o["num_vis_per_wplane"], o["num_vis_per_grid"],
        o["avg_wsupport_per_grid"], o["avg_wplane_per_grid"])
    o["norm"] = nrm
    o["num_skipped"] = sk
    return o


def check_against(got, want):
    for k in ("num_vis_per_wsupport", "num_vis_per_wplane",
              "num_vis_per_grid", "avg_wsupport_per_grid",
              "avg_wplane_per_grid"):
        assert np.array_equal(got[k], want[k]), k
    assert got["num_skipped"] == want["num_skipped"]
    assert abs(got["norm"] - want["norm"]) <= 1e-12 * abs(want["norm"])
    assert rel_rms(got["grid"], want["grid"]) <= TOL_F


def zero_init(w):
    g = w["grid_size"]
    ns, npl = O.diagnostics_sizes(w)
    return dict(grid=np.zeros(2 * g * g, np.float32), norm=0.0,
                num_vis_per_wsupport=np.zeros(ns, np.int64),
                num_vis_per_wplane=np.zeros(npl, np.int64),
                num_vis_per_grid=np.zeros(g * g, np.int64),
                avg_wsupport_per_grid=np.zeros(g * g, np.float32),
                avg_wplane_per_grid=np.zeros(g * g, np.float32))


def test_diagnostics_matches_reference_golden():
    """Edge-case points (footprints on and past every edge, planes past the
    last one, up to plane 10^6, half-way roundings) with every array
    starting from non-zero contents: the reference's outputs."""
    inputs, init, out = load_diag_golden("diag_edges_f")
    check_against(run_gpu(inputs, init), out)


def test_diagnostics_matches_oracle_on_a_synthetic_job():
    w = W.plain_small(seed=6).numpy()
    for k in ("uu", "vv", "ww", "weight"):
        w[k] = w[k][:120000]
    w["vis"] = w["vis"][:240000]
    for k in ("conv_func", "uu", "vv", "ww", "vis", "weight"):
        w[k] = np.asarray(w[k], np.float32)
    w["cell_size_rad"] = float(np.float32(w["cell_size_rad"]))
    w["w_scale"] = float(np.float32(w["w_scale"]))
    got = run_gpu(w, zero_init(w))
    want = O.diagnostics_f(w)
    check_against(got, want)
    assert got["num_vis_per_grid"].sum() > 0


def test_diagnostics_empty_job_touches_only_the_skip_count():
    inputs, init, _ = load_diag_golden("diag_edges_f")
    w = dict(inputs)
    for k in ("uu", "vv", "ww", "weight"):
        w[k] = w[k][:0]
    w["vis"] = w["vis"][:0]
    got = run_gpu(w, init)
    assert got["num_skipped"] == 0 and got["norm"] == init["norm"]
    for k, v in init.items():
        if k != "norm":
            assert np.array_equal(got[k], v), k


def test_diagnostics_refuses_unusable_plane_index():
    """A w whose plane index round(sqrt(|w| w_scale)) is 2^24 or more (the
    reference would index num_vis_per_wplane out of any sane array): the
    call fails before anything is written."""
    inputs, init, _ = load_diag_golden("diag_edges_f")
    w = dict(inputs)
    w["ww"] = np.array(w["ww"], copy=True)
    w["ww"][3] = 1e30
    o = {k: (v if k == "norm" else np.array(v, copy=True))
         for k, v in init.items()}
    with pytest.raises(fg.GridderError) as e:
        run_gpu(w, o, copy=False)
    assert e.value.status == _lib.ERR_INVALID_ARGUMENT
    for k, v in init.items():
        if k != "norm":
            assert np.array_equal(o[k], v), k
