"""Generates the golden fixtures in this directory from the reference's own
gridder (oskar_grid_wproj.c compiled unmodified into
oracle/_ref/libref_gridder.so by oracle/Makefile).

Run from the repository root, where the reference sources are available:
    make -C oracle && python tests/golden/make_golden.py

Each .npz holds the inputs in the reference's argument convention and the
reference's outputs (grid, norm, num_skipped).  The fixtures pin both the
oracle restatement (bit-exact) and the GPU gridder (tolerance) without the
reference being present.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from fpga_gridding_b200 import workloads as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def edge_case_inputs(seed=7):
    """Hand-placed points on every branch of the reference's placement:
    half-way rounding of cell and offset, footprint exactly touching each
    grid edge and one cell past it, w-plane clamping, w > 0 conjugation,
    w = 0, plus random fill.  grid_scale = grid_size * cell = 1 so positions
    are in cells; w_scale = 1 so plane = round(sqrt(|w|))."""
    rng = np.random.default_rng(seed)
    g = 64
    support = np.array([1, 2, 3, 3], dtype=np.int32)
    os_ = 4
    csh = os_ * 3 + 2 + 1 + 2
    pts = []  # (u, v, w)  with pos_u = -u, pos_v = v
    for u in (0.5, -0.5, 1.5, -1.5, 2.5, 0.125, 0.375, 0.625, -0.375,
              -0.625, 0.875, 0.3749999, 0.3750001):
        for w in (0.0, 2.25, -2.25, 5.0, -100.0):
            pts.append((u, u * 0.5 - 0.25, w))
    centre = g // 2
    for s_idx, w in enumerate((0.0, 1.0, 4.0, 9.0)):
        s = int(support[min(s_idx, 3)])
        # footprint touching the low edge (kept) and one past (skipped)
        for d in (0, 1):
            gu = s - d
            pts.append((-(gu - centre), 0.0, w))
            pts.append((0.0, (gu - centre), -w))
            gu = g - 1 - s + d
            pts.append((-(gu - centre), 0.0, w))
            pts.append((0.0, (gu - centre), w))
    # far outside and huge w
    pts += [(1e9, 0.0, 0.0), (0.0, -1e9, 1.0), (0.0, 0.0, 1e12)]
    n_rand = 400
    ru = rng.uniform(-30, 30, n_rand)
    rv = rng.uniform(-30, 30, n_rand)
    rw = rng.uniform(-20, 20, n_rand)
    pts += list(zip(ru, rv, rw))
    a = np.array(pts, dtype=np.float64)
    n = a.shape[0]
    vis = rng.normal(size=2 * n)
    cube = rng.normal(size=len(support) * csh * csh * 2)
    return dict(num_w_planes=len(support), support=support, oversample=os_,
                conv_size_half=csh, conv_func=cube, uu=a[:, 0].copy(),
                vv=a[:, 1].copy(), ww=a[:, 2].copy(), vis=vis,
                weight=np.ones(n), cell_size_rad=1.0 / g, w_scale=1.0,
                grid_size=g)


def odd_oversample_inputs(seed=11):
    """Oversample 3 (offsets in [-2, 2]) and a zero-support plane."""
    rng = np.random.default_rng(seed)
    g = 48
    support = np.array([0, 1, 2, 4], dtype=np.int32)
    os_ = 3
    csh = os_ * 4 + 2 + 1
    n = 600
    uu = rng.uniform(-18, 18, n)
    vv = rng.uniform(-18, 18, n)
    ww = rng.uniform(-25, 25, n)
    return dict(num_w_planes=len(support), support=support, oversample=os_,
                conv_size_half=csh, conv_func=rng.normal(size=4 * csh * csh * 2),
                uu=uu, vv=vv, ww=ww, vis=rng.normal(size=2 * n),
                weight=np.ones(n), cell_size_rad=1.0 / g, w_scale=1.0,
                grid_size=g)


def synth_small_inputs(num_points=10000):
    """A scaled plain W-projection job: 16 stations in a 500 m disk, 84
    samples (10080 visibilities, the first num_points kept), 8 planes with
    support 2 -> 6, oversample 4, grid 128."""
    wl = W.plain_small(seed=3, num_stations=16, num_times=84, grid_size=128,
                       num_w_planes=8)
    w = wl.numpy()
    support = W.support_ramp(8, 2, 6)
    csh = W.min_conv_size_half(support, 4) + 1
    cube = W.analytic_kernel_cube(support, 4, csh).numpy()
    uv_max = max(np.abs(w["uu"]).max(), np.abs(w["vv"]).max())
    cell = (128 // 2 - 6 - 2) / (128 * uv_max)
    sel = slice(0, num_points)
    return dict(num_w_planes=8, support=support, oversample=4,
                conv_size_half=csh, conv_func=cube, uu=w["uu"][sel].copy(),
                vv=w["vv"][sel].copy(), ww=w["ww"][sel].copy(),
                vis=w["vis"][: 2 * num_points].copy(),
                weight=np.ones(num_points), cell_size_rad=float(cell),
                w_scale=float(w["w_scale"]), grid_size=128)


def ones_inputs():
    """Known answer: every kernel tap and visibility is 1 + 0i (the
    reference's FAKE_VIS_VALUES / FAKE_KERNEL_VALUES mode, Defines.h:37-38):
    each kept point adds 1 to every cell of its footprint and (2S+1)^2 to
    norm."""
    d = synth_small_inputs(2000)
    cube = np.zeros_like(d["conv_func"])
    cube[0::2] = 1.0
    d["conv_func"] = cube
    vis = np.zeros_like(d["vis"])
    vis[0::2] = 1.0
    d["vis"] = vis
    return d


def weights_inputs(seed=13):
    """Uniform-weighting case (utils/oskar_grid_weights.c): grid_scale = 1
    so positions are in cells; half-way positions, the first and last cell
    of each axis and one past them, far-outside points, and a dense cluster
    of points with non-integer weights so that many cells sum several
    weights (their order matters).  The weights grid and weight_out start
    from random values: the write accumulates and the read leaves skipped
    points' outputs alone."""
    rng = np.random.default_rng(seed)
    g = 64
    pts = []  # (u, v): pos_u = -u, pos_v = v
    for u in (0.5, -0.5, 1.5, -1.5, 2.5, -2.5, 0.49999997, 0.50000003):
        pts.append((u, -u))
    for e in (32.0, 32.4, 32.5, -31.0, -31.4, -31.5, 1e9, -1e9):
        pts.append((e, 0.0))
        pts.append((0.0, -e))
    n_rand = 3000
    ru = rng.normal(0.0, 4.0, n_rand)
    rv = rng.normal(0.0, 4.0, n_rand)
    pts += list(zip(ru, rv))
    a = np.array(pts, dtype=np.float64)
    n = a.shape[0]
    return dict(uu=a[:, 0].copy(), vv=a[:, 1].copy(),
                weight=rng.uniform(0.1, 3.0, n), cell_size_rad=1.0 / g,
                grid_size=g, grid=rng.uniform(0.0, 2.0, g * g),
                weight_out=rng.uniform(-1.0, 1.0, n))


def save_weights(name, inputs, single):
    """Runs the reference's oskar_grid_weights_write then _read on the
    inputs and stores inputs and outputs."""
    import ctypes as C
    ref = O.reference_lib()
    if ref is None:
        raise SystemExit("build oracle/_ref first (make -C oracle)")
    real = np.float32 if single else np.float64
    t = "f" if single else "d"
    a = {k: np.ascontiguousarray(inputs[k], dtype=real)
         for k in ("uu", "vv", "weight", "grid", "weight_out")}
    cell = real(inputs["cell_size_rad"])
    g = inputs["grid_size"]
    n = a["uu"].size
    grid = a["grid"].copy()
    wout = a["weight_out"].copy()
    sk_w = C.c_size_t(0)
    sk_r = C.c_size_t(0)
    getattr(ref, "ref_oskar_grid_weights_write_" + t)(
        n, a["uu"].ctypes.data, a["vv"].ctypes.data, a["weight"].ctypes.data,
        cell, g, C.byref(sk_w), grid.ctypes.data)
    getattr(ref, "ref_oskar_grid_weights_read_" + t)(
        n, a["uu"].ctypes.data, a["vv"].ctypes.data, a["weight"].ctypes.data,
        wout.ctypes.data, cell, g, C.byref(sk_r), grid.ctypes.data)
    np.savez_compressed(
        os.path.join(OUT, name + ".npz"), cell_size_rad=np.asarray(cell),
        grid_size=g, single=single, out_grid=grid, out_weight=wout,
        out_skipped_write=sk_w.value, out_skipped_read=sk_r.value, **a)
    print(f"{name}: n={n} skipped={sk_w.value}/{sk_r.value}")


def save(name, inputs, single):
    ref = O.reference_lib()
    if ref is None:
        raise SystemExit("build oracle/_ref first (make -C oracle)")
    real = np.float32 if single else np.float64
    fn = ref.ref_oskar_grid_wproj_f if single else ref.ref_oskar_grid_wproj_d
    if single:
        # The shipped FP32 reference always processes exactly 10000 points.
        assert len(inputs["uu"]) == 10000
    skipped, norm, grid = O.grid(fn, inputs, real)
    arrays = {k: np.asarray(v, dtype=real) for k, v in inputs.items()
              if k in ("conv_func", "uu", "vv", "ww", "vis", "weight")}
    np.savez_compressed(
        os.path.join(OUT, name + ".npz"), support=inputs["support"],
        num_w_planes=inputs["num_w_planes"], oversample=inputs["oversample"],
        conv_size_half=inputs["conv_size_half"],
        cell_size_rad=np.asarray(inputs["cell_size_rad"], dtype=real),
        w_scale=np.asarray(inputs["w_scale"], dtype=real),
        grid_size=inputs["grid_size"], out_grid=grid, out_norm=norm,
        out_skipped=skipped, single=single, **arrays)
    print(f"{name}: n={len(inputs['uu'])} skipped={skipped} norm={norm:.17g}")


def save_diagnostics(name, inputs, seed=17):
    """Runs the reference's oskar_grid_wproj_f_diagnostics on the inputs
    (as float) with every in/out array starting from random contents (the
    counts and per-cell sums from small integers, so the accumulation stays
    exact; the plane histogram random over its first 64 entries, zero
    beyond) and stores inputs, starting contents and outputs."""
    rng = np.random.default_rng(seed)
    w = dict(inputs)
    for k in ("conv_func", "uu", "vv", "ww", "vis", "weight"):
        w[k] = np.asarray(inputs[k], dtype=np.float32)
    w["cell_size_rad"] = float(np.float32(inputs["cell_size_rad"]))
    w["w_scale"] = float(np.float32(inputs["w_scale"]))
    g = w["grid_size"]
    ns, npl = O.diagnostics_sizes(w)
    init = dict(grid=rng.normal(size=2 * g * g).astype(np.float32),
                norm=0.5,
                num_vis_per_wsupport=rng.integers(0, 5, ns).astype(np.int64),
                num_vis_per_wplane=np.concatenate([
                    rng.integers(0, 5, min(npl, 64)),
                    np.zeros(max(0, npl - 64), np.int64)]).astype(np.int64),
                num_vis_per_grid=rng.integers(0, 5, g * g).astype(np.int64),
                avg_wsupport_per_grid=rng.integers(0, 50, g * g).astype(
                    np.float32),
                avg_wplane_per_grid=rng.uniform(size=g * g).astype(
                    np.float32))
    out = O.diagnostics_f(w, use_reference=True, init=init)
    arrays = {k: w[k] for k in ("conv_func", "uu", "vv", "ww", "vis",
                                "weight")}
    np.savez_compressed(
        os.path.join(OUT, name + ".npz"), support=inputs["support"],
        num_w_planes=inputs["num_w_planes"], oversample=inputs["oversample"],
        conv_size_half=inputs["conv_size_half"],
        cell_size_rad=np.asarray(w["cell_size_rad"], dtype=np.float32),
        w_scale=np.asarray(w["w_scale"], dtype=np.float32),
        grid_size=g, single=True, **arrays,
        **{"init_" + k: np.asarray(v) for k, v in init.items()},
        **{"out_" + k: np.asarray(v) for k, v in out.items()})
    print(f"{name}: n={len(w['uu'])} skipped={out['num_skipped']} "
          f"planes hist={npl}")


def main():
    save("edges_d", edge_case_inputs(), single=False)
    save("odd_oversample_d", odd_oversample_inputs(), single=False)
    save("synth_small_d", synth_small_inputs(), single=False)
    save("synth_small_f", synth_small_inputs(), single=True)
    save("ones_d", ones_inputs(), single=False)
    save_weights("weights_d", weights_inputs(), single=False)
    save_weights("weights_f", weights_inputs(), single=True)
    save_diagnostics("diag_edges_f", edge_case_inputs())


if __name__ == "__main__":
    main()
