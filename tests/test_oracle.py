"""The CPU oracle is pinned to the reference: bit-exact against the
reference's own gridder compiled from its sources (oracle/_ref) and against
the golden fixtures generated from it."""
import numpy as np
import pytest

from conftest import golden_names, load_golden, load_weights_golden
from fpga_gridding_b200 import workloads as W


@pytest.fixture(scope="module")
def small():
    return W.plain_small().numpy()


@pytest.fixture(scope="module")
def ref(oracle):
    lib = oracle.reference_lib()
    if lib is None:
        pytest.skip("reference not compiled here (oracle/_ref missing)")
    return lib


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_golden_bit_exact(oracle, name):
    inputs, out = load_golden(name)
    fn = oracle.grid_f if out["single"] else oracle.grid_d
    skipped, norm, grid = fn(inputs)
    assert skipped == out["skipped"]
    assert norm == out["norm"]
    assert np.array_equal(grid, out["grid"])


def test_oracle_d_matches_reference_full_small_config(oracle, ref, small):
    s1, n1, g1 = oracle.grid(ref.ref_oskar_grid_wproj_d, small, np.float64)
    s2, n2, g2 = oracle.grid_d(small)
    assert (s1, n1) == (s2, n2)
    assert np.array_equal(g1, g2)


def test_oracle_f_matches_reference_on_10000_point_slices(oracle, ref, small):
    # The shipped FP32 reference grids exactly 10000 points per call
    # (oskar_grid_wproj.c:155); compare slice by slice, accumulating.
    g = small["grid_size"]
    g1 = np.zeros(2 * g * g, np.float32)
    g2 = np.zeros(2 * g * g, np.float32)
    n1 = n2 = 0.0
    for start in (0, 10000, 120000, 230000):
        part = dict(small)
        for k in ("uu", "vv", "ww", "weight"):
            part[k] = small[k][start:start + 10000]
        part["vis"] = small["vis"][2 * start:2 * (start + 10000)]
        s1, n1, g1 = oracle.grid(ref.ref_oskar_grid_wproj_f, part, np.float32,
                                 g1, n1)
        s2, n2, g2 = oracle.grid_f(part, g2, n2)
        assert s1 == s2
    assert n1 == n2
    assert np.array_equal(g1, g2)


def test_banded_threads_bit_identical_to_serial(oracle, small):
    s1, n1, g1 = oracle.grid_d(small)
    for t in (1, 3, 8):
        s2, n2, g2 = oracle.grid_d(small, threads=t)
        assert (s1, n1) == (s2, n2)
        assert np.array_equal(g1, g2)
    inputs, _ = load_golden("edges_d")
    s1, n1, g1 = oracle.grid_d(inputs)
    s2, n2, g2 = oracle.grid_d(inputs, threads=5)
    assert (s1, n1) == (s2, n2) and np.array_equal(g1, g2)
    fs1, fn1, fg1 = oracle.grid_f(small)
    fs2, fn2, fg2 = oracle.grid_f(small, threads=4)
    assert (fs1, fn1) == (fs2, fn2) and np.array_equal(fg1, fg2)


def test_known_answer_all_ones(oracle):
    """FAKE_VIS_VALUES / FAKE_KERNEL_VALUES mode (Defines.h:37-38): every
    kept point adds 1 to each footprint cell and (2S+1)^2 to norm."""
    inputs, out = load_golden("ones_d")
    p = oracle.place(inputs)
    keep = p["skipped"] == 0
    s = inputs["support"][p["plane"][keep]]
    assert out["norm"] == float(np.sum((2 * s + 1) ** 2))
    g = inputs["grid_size"]
    expect = np.zeros((g, g))
    for gu, gv, sp in zip(p["gu"][keep], p["gv"][keep], s):
        expect[gv - sp:gv + sp + 1, gu - sp:gu + sp + 1] += 1.0
    grid = out["grid"].reshape(g, g, 2)
    assert np.array_equal(grid[..., 0], expect)
    assert not grid[..., 1].any()


def test_placement_edge_cases(oracle):
    inputs, out = load_golden("edges_d")
    p = oracle.place(inputs)
    assert int(p["skipped"].sum()) == out["skipped"]
    # half-way cell rounding is away from zero: u = 0.5 -> pos_u = -0.5
    # -> round -> -1 -> grid_u = 31
    assert p["gu"][0] == 31
    # plane clamp: w = -100 -> round(10) clamps to the last plane (3)
    assert p["raw_plane"][4] == 10 and p["plane"][4] == 3
    # conjugation only for w > 0
    assert p["conj"][1] == -1 and p["conj"][0] == 1 and p["conj"][2] == 1
    # offsets stay within [-os/2, os/2]
    assert np.abs(p["off_u"][p["skipped"] == 0]).max() <= 2


def test_float_coordinates_differ_from_double_only_rarely(oracle, small):
    pd = oracle.place(small)
    pf = oracle.place(small, single=True)
    diff = sum(int((pd[k] != pf[k]).sum()) for k in ("gu", "gv", "plane"))
    assert diff < small["uu"].size * 1e-3


def test_weights_restatement_matches_reference(oracle, ref, small):
    import ctypes as C
    n = small["uu"].size
    g = small["grid_size"]
    for real, t in ((np.float64, "d"), (np.float32, "f")):
        uu = small["uu"].astype(real)
        vv = small["vv"].astype(real)
        w1 = np.ones(n, real)
        outs = []
        for lib, prefix in ((ref, "ref_oskar_"), (oracle.oracle_lib(), "orc_")):
            grid = np.zeros(g * g, real)
            sk = C.c_size_t(0)
            getattr(lib, prefix + "grid_weights_write_" + t)(
                n, uu.ctypes.data, vv.ctypes.data, w1.ctypes.data,
                small["cell_size_rad"], g, C.byref(sk), grid.ctypes.data)
            wout = np.zeros(n, real)
            sk2 = C.c_size_t(0)
            getattr(lib, prefix + "grid_weights_read_" + t)(
                n, uu.ctypes.data, vv.ctypes.data, w1.ctypes.data,
                wout.ctypes.data, small["cell_size_rad"], g, C.byref(sk2),
                grid.ctypes.data)
            outs.append((sk.value, sk2.value, grid, wout))
        assert outs[0][:2] == outs[1][:2]
        assert np.array_equal(outs[0][2], outs[1][2])
        assert np.array_equal(outs[0][3], outs[1][3])


@pytest.mark.parametrize("name", ["weights_d", "weights_f"])
def test_weights_oracle_matches_golden_bit_exact(oracle, name):
    z = load_weights_golden(name)
    sk_w, grid, sk_r, wout = oracle.weights(
        z["uu"], z["vv"], z["weight"], z["cell_size_rad"], int(z["grid_size"]),
        z["grid"], z["weight_out"], single=bool(z["single"]))
    assert sk_w == int(z["out_skipped_write"])
    assert sk_r == int(z["out_skipped_read"])
    assert np.array_equal(grid, z["out_grid"])
    assert np.array_equal(wout, z["out_weight"])
    # Cells summing several non-integer weights are present, so the
    # fixture pins the summation order.
    cells = np.round(-z["uu"] * z["grid_size"] * z["cell_size_rad"])
    assert np.unique(cells).size < cells.size // 4


def test_weights_restatement_matches_reference_random_weights(oracle, ref,
                                                              small):
    rng = np.random.default_rng(21)
    n = small["uu"].size
    g = small["grid_size"]
    for single in (False, True):
        args = (small["uu"], small["vv"], rng.uniform(0.1, 2.0, n),
                small["cell_size_rad"], g, rng.uniform(0, 1, g * g),
                rng.uniform(-1, 1, n))
        a = oracle.weights(*args, single=single)
        b = oracle.weights(*args, single=single, use_reference=True)
        assert a[0] == b[0] and a[2] == b[2]
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[3], b[3])


def test_weights_parallel_harness_matches_serial_for_unit_weights(oracle,
                                                                 small):
    g = small["grid_size"]
    n = small["uu"].size
    ones = np.ones(n)
    for use_ref in (False, True):
        secs, sk_w, grid, sk_r, wout = oracle.time_weights_parallel(
            small["uu"], small["vv"], ones, small["cell_size_rad"], g, 3,
            use_ref)
        s_w, g1, s_r, w1 = oracle.weights(
            small["uu"], small["vv"], ones, small["cell_size_rad"], g,
            np.zeros(g * g), np.zeros(n), single=True)
        assert secs > 0 and (sk_w, sk_r) == (s_w, s_r)
        assert np.array_equal(grid, g1) and np.array_equal(wout, w1)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_scale_coords_restatement_matches_reference(oracle, ref, dtype):
    if oracle.reference_ingest_lib() is None:
        pytest.skip("reference ingest library not built")
    rng = np.random.default_rng(8)
    uu, vv, ww = (rng.normal(0.0, 3000.0, 50000).astype(dtype)
                  for _ in range(3))
    for f in (50e6, 149.97e6, 1.4204e9):
        a = oracle.scale_coords(f, uu, vv, ww)
        b = oracle.scale_coords(f, uu, vv, ww, use_reference=True)
        for x, y in zip(a, b):
            assert x.dtype == dtype and np.array_equal(x, y)


def test_degrid_oracle_is_the_adjoint_of_the_gridder(oracle, small):
    """<G v, g> == <v, G^H g> for the oracle's gridder G and degridder G^H
    on the plain_small job and a random complex grid."""
    rng = np.random.default_rng(1)
    g = small["grid_size"]
    gr = rng.normal(size=2 * g * g)
    sk, vis_adj = oracle.degrid_d(small, gr)
    s1, _, gv = oracle.grid_d(small)
    assert sk == s1
    v = np.asarray(small["vis"], np.float64)
    lhs = np.vdot(gr[0::2] + 1j * gr[1::2], gv[0::2] + 1j * gv[1::2])
    rhs = np.vdot(vis_adj[0::2] + 1j * vis_adj[1::2], v[0::2] + 1j * v[1::2])
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_parallel_timing_harness_sums_to_serial(oracle, small):
    secs, sk, nrm, grid = oracle.time_parallel(small, False, 3, False,
                                               want_grid=True)
    s1, n1, g1 = oracle.grid_d(small)
    assert secs > 0 and sk == s1
    assert abs(nrm - n1) <= 1e-12 * abs(n1)
    assert oracle.rel_rms(grid, g1) < 1e-13


def test_weighted_oracle_with_unit_weights_is_the_reference(oracle, ref):
    """The weighted restatement (the reference tiled CUDA gridder's
    weighting) with unit weights is the reference's own oskar_grid_wproj_d,
    bit for bit."""
    w = W.plain_small(num_stations=24, num_times=40, grid_size=256,
                      num_w_planes=8).numpy()
    w["weight"] = np.ones_like(w["weight"])
    s1, n1, g1 = oracle.grid(ref.ref_oskar_grid_wproj_d, w, np.float64)
    s2, n2, g2 = oracle.grid_weighted_d(w)
    assert (s1, n1) == (s2, n2)
    assert np.array_equal(g1, g2)


def test_weighted_oracle_scales_each_visibility(oracle):
    """Random weights: the grid equals the unweighted gridder's on the
    visibilities times their weights (the same products, the same order);
    weights of exactly 2 double the norm exactly."""
    w = W.plain_small(num_stations=24, num_times=40, grid_size=256,
                      num_w_planes=8).numpy()
    rng = np.random.default_rng(4)
    w["weight"] = rng.uniform(0.25, 4.0, len(w["uu"]))
    s1, n1, g1 = oracle.grid_weighted_d(w)
    scaled = dict(w)
    scaled["vis"] = (w["vis"].reshape(-1, 2) *
                     w["weight"][:, None]).reshape(-1)
    s2, _, g2 = oracle.grid_d(scaled)
    assert s1 == s2 and np.array_equal(g1, g2)
    two = dict(w)
    two["weight"] = np.full(len(w["uu"]), 2.0)
    _, n_two, _ = oracle.grid_weighted_d(two)
    _, n_one, _ = oracle.grid_d(w)
    assert n_two == 2.0 * n_one


def _diag_equal(a, b):
    for k in ("grid", "num_vis_per_wsupport", "num_vis_per_wplane",
              "num_vis_per_grid", "avg_wsupport_per_grid",
              "avg_wplane_per_grid"):
        assert np.array_equal(a[k], b[k]), k
    assert a["norm"] == b["norm"]
    assert a["num_skipped"] == b["num_skipped"]


def test_diagnostics_oracle_matches_golden_bit_exact(oracle):
    """oskar_grid_wproj_f_diagnostics (oskar_grid_wproj.c:245-370),
    restated, against the reference's own outputs on the edge-case points
    (skipped footprints, planes past the last one, half-way roundings) with
    every in/out array starting from non-zero contents."""
    from conftest import load_diag_golden
    inputs, init, out = load_diag_golden("diag_edges_f")
    _diag_equal(oracle.diagnostics_f(inputs, init=init), out)


def test_diagnostics_oracle_matches_reference(oracle, ref, small):
    part = dict(small)
    for k in ("uu", "vv", "ww", "weight"):
        part[k] = small[k][:30000]
    part["vis"] = small["vis"][:60000]
    _diag_equal(oracle.diagnostics_f(part),
                oracle.diagnostics_f(part, use_reference=True))


def test_diagnostics_grid_is_the_float_gridder(oracle, small):
    """The diagnostics variant grids exactly as oskar_grid_wproj_f (without
    its fixed 10000-point loop), and its counts add up: one count per point
    in each histogram, one per tap of a kept point per cell."""
    part = dict(small)
    for k in ("uu", "vv", "ww", "weight"):
        part[k] = small[k][:20000]
    part["vis"] = small["vis"][:40000]
    d = oracle.diagnostics_f(part)
    s, n, g = oracle.grid_f(part)
    assert d["num_skipped"] == s and d["norm"] == n
    assert np.array_equal(d["grid"], g)
    assert d["num_vis_per_wsupport"].sum() == 20000
    assert d["num_vis_per_wplane"].sum() == 20000
    p = oracle.place(part, single=True)
    kept = p["skipped"] == 0
    sup = np.asarray(part["support"])[p["plane"][kept]]
    assert d["num_vis_per_grid"].sum() == int(((2 * sup + 1) ** 2).sum())
    assert not d["avg_wplane_per_grid"].any()
