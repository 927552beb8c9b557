"""ctypes front end for the CPU checker libraries.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg import this module.  It wraps:

  liboracle.so             the C restatement in oracle.c (always built), and
  _ref/libref_gridder.so   the reference's oskar_grid_wproj.c and
                           oskar_grid_weights.c compiled unmodified
                           (present where the reference sources were
                           available at build time).
  _ref/libref_ingest.so    the reference's read_vis.c (read_coords,
                           scale_coords) and OSKAR binary file library,
                           compiled unmodified (same condition).

Build both with `make -C oracle`.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libref_gridder.so")
REF_INGEST_SO = os.path.join(HERE, "_ref", "libref_ingest.so")

_P = C.c_void_p
_SZ = C.c_size_t

_GRID_ARGS_D = [_SZ, _P, C.c_int, C.c_int, _P, _SZ, _P, _P, _P, _P, _P,
                C.c_double, C.c_double, C.c_int, _P, _P, _P]
_GRID_ARGS_F = [_SZ, _P, C.c_int, C.c_int, _P, _SZ, _P, _P, _P, _P, _P,
                C.c_float, C.c_float, C.c_int, _P, _P, _P]
_DIAG_ARGS = _GRID_ARGS_F + [_P] * 5
GRID_FN_D = C.CFUNCTYPE(None, *_GRID_ARGS_D)
GRID_FN_F = C.CFUNCTYPE(None, *_GRID_ARGS_F)

_oracle = None
_ref = None


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and _ref/ where the reference sources exist)."""
    out = subprocess.run(["make", "-C", HERE, "all"], capture_output=True,
                         text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _declare(lib, prefix):
    for suffix, args in (("grid_wproj_d", _GRID_ARGS_D),
                         ("grid_wproj_f", _GRID_ARGS_F)):
        fn = getattr(lib, prefix + suffix)
        fn.argtypes = args
        fn.restype = None
    return lib


def oracle_lib():
    """The C restatement (builds it on first use if missing)."""
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build()
        lib = _declare(C.CDLL(ORACLE_SO), "orc_")
        pl = [_SZ, _P, C.c_int, _SZ, _P, _P, _P]
        lib.orc_vis_place_d.argtypes = pl + [C.c_double, C.c_double, C.c_int] + [_P] * 8
        lib.orc_vis_place_f.argtypes = pl + [C.c_float, C.c_float, C.c_int] + [_P] * 8
        lib.orc_vis_place_d.restype = lib.orc_vis_place_f.restype = None
        lib.orc_grid_wproj_weighted_d.argtypes = _GRID_ARGS_D
        lib.orc_grid_wproj_weighted_d.restype = None
        lib.orc_grid_wproj_d_banded.argtypes = _GRID_ARGS_D + [C.c_int]
        lib.orc_grid_wproj_f_banded.argtypes = _GRID_ARGS_F + [C.c_int]
        lib.orc_count_taps_d.argtypes = [_SZ, _P, C.c_int, _SZ, _P, _P, _P,
                                         C.c_double, C.c_double, C.c_int]
        lib.orc_count_taps_d.restype = C.c_uint64
        for t, fa in (("d", (C.c_double, _GRID_ARGS_D)),
                      ("f", (C.c_float, _GRID_ARGS_F))):
            fn = getattr(lib, "orc_time_parallel_" + t)
            fn.argtypes = [_P, C.c_int, _SZ] + fa[1][:13] + [_P, _P, _P]
            fn.restype = C.c_double
            w = getattr(lib, "orc_grid_weights_write_" + t)
            w.argtypes = [_SZ, _P, _P, _P, fa[0], C.c_int, _P, _P]
            r = getattr(lib, "orc_grid_weights_read_" + t)
            r.argtypes = [_SZ, _P, _P, _P, _P, fa[0], C.c_int, _P, _P]
            w.restype = r.restype = None
        lib.orc_time_weights_parallel_f.argtypes = [
            _P, _P, C.c_int, _SZ, _P, _P, _P, C.c_float, C.c_int, _P, _P,
            _P, _P]
        lib.orc_time_weights_parallel_f.restype = C.c_double
        lib.orc_degrid_wproj_d.argtypes = [
            _SZ, _P, C.c_int, C.c_int, _P, _SZ, _P, _P, _P, C.c_double,
            C.c_double, C.c_int, _P, _P, _P]
        lib.orc_degrid_wproj_d.restype = None
        lib.orc_scale_coords.argtypes = [C.c_double, C.c_int, _SZ, _P, _P, _P]
        lib.orc_scale_coords.restype = None
        lib.orc_grid_wproj_f_diagnostics.argtypes = _DIAG_ARGS
        lib.orc_grid_wproj_f_diagnostics.restype = None
        _oracle = lib
    return _oracle


def reference_lib():
    """The reference compiled from its own sources, or None if not built."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            return None
        lib = _declare(C.CDLL(REF_SO), "ref_oskar_")
        for t, real in (("d", C.c_double), ("f", C.c_float)):
            w = getattr(lib, "ref_oskar_grid_weights_write_" + t)
            w.argtypes = [_SZ, _P, _P, _P, real, C.c_int, _P, _P]
            r = getattr(lib, "ref_oskar_grid_weights_read_" + t)
            r.argtypes = [_SZ, _P, _P, _P, _P, real, C.c_int, _P, _P]
            w.restype = r.restype = None
        lib.ref_oskar_grid_wproj_f_diagnostics.argtypes = _DIAG_ARGS
        lib.ref_oskar_grid_wproj_f_diagnostics.restype = None
        _ref = lib
    return _ref


_ref_ingest = None


def reference_ingest_lib():
    """The reference's read_vis.c + OSKAR binary library, or None."""
    global _ref_ingest
    if _ref_ingest is None:
        if not os.path.exists(REF_INGEST_SO):
            return None
        lib = C.CDLL(REF_INGEST_SO)
        lib.ref_scale_coords.argtypes = [C.c_double, C.c_int, _SZ, _P, _P, _P]
        lib.ref_scale_coords.restype = None
        _ref_ingest = lib
    return _ref_ingest


def scale_coords(freq_hz: float, uu, vv, ww, use_reference: bool = False):
    """Metres to wavelengths as utils/read_vis.c:51-73 (restated, or the
    reference's own function): returns scaled copies in the arrays'
    precision (float32 or float64)."""
    a = [np.array(x, copy=True) for x in (uu, vv, ww)]
    dbl = a[0].dtype == np.float64
    assert all(x.dtype == a[0].dtype and x.flags.c_contiguous for x in a)
    if use_reference:
        lib = reference_ingest_lib()
        if lib is None:
            raise RuntimeError("reference ingest library not built")
        # OSKAR_DOUBLE = 0x08, OSKAR_SINGLE = 0x04
        # (utils/binary/oskar_binary_data_types.h:52-55)
        lib.ref_scale_coords(freq_hz, 0x08 if dbl else 0x04, a[0].size,
                             _ptr(a[0]), _ptr(a[1]), _ptr(a[2]))
    else:
        oracle_lib().orc_scale_coords(freq_hz, int(dbl), a[0].size,
                                      _ptr(a[0]), _ptr(a[1]), _ptr(a[2]))
    return a


def _ptr(a):
    return a.ctypes.data_as(_P) if a is not None else None


def _arrays(w: dict, dtype):
    """Contiguous arrays of one dtype from a Workload.numpy() dict."""
    conv = lambda k: np.ascontiguousarray(w[k], dtype=dtype)
    return dict(support=np.ascontiguousarray(w["support"], dtype=np.int32),
                conv_func=conv("conv_func"), uu=conv("uu"), vv=conv("vv"),
                ww=conv("ww"), vis=conv("vis"), weight=conv("weight"))


def grid(fn, w: dict, dtype, grid_arr=None, norm: float = 0.0,
         threads: int | None = None):
    """Call a gridding function with the reference's signature on the arrays
    of `w`.  Returns (num_skipped, norm, grid)."""
    a = _arrays(w, dtype)
    g = w["grid_size"]
    if grid_arr is None:
        grid_arr = np.zeros(2 * g * g, dtype=dtype)
    skipped = C.c_size_t(0)
    nrm = C.c_double(norm)
    args = [w["num_w_planes"], _ptr(a["support"]), w["oversample"],
            w["conv_size_half"], _ptr(a["conv_func"]), a["uu"].shape[0],
            _ptr(a["uu"]), _ptr(a["vv"]), _ptr(a["ww"]), _ptr(a["vis"]),
            _ptr(a["weight"]), w["cell_size_rad"], w["w_scale"], g,
            C.byref(skipped), C.byref(nrm), _ptr(grid_arr)]
    if threads is not None:
        args.append(threads)
    fn(*args)
    return skipped.value, nrm.value, grid_arr


def grid_d(w, grid_arr=None, norm=0.0, threads=None):
    """Oracle FP64 gridding (banded threads when `threads` is given)."""
    lib = oracle_lib()
    fn = lib.orc_grid_wproj_d if threads is None else lib.orc_grid_wproj_d_banded
    return grid(fn, w, np.float64, grid_arr, norm, threads)


def grid_weighted_d(w, grid_arr=None, norm=0.0):
    """Oracle FP64 gridding with each visibility scaled by its weight (the
    reference tiled CUDA gridder's weighting)."""
    return grid(oracle_lib().orc_grid_wproj_weighted_d, w, np.float64,
                grid_arr, norm)


def grid_f(w, grid_arr=None, norm=0.0, threads=None):
    """Oracle FP32 gridding with the reference's float coordinates."""
    lib = oracle_lib()
    fn = lib.orc_grid_wproj_f if threads is None else lib.orc_grid_wproj_f_banded
    return grid(fn, w, np.float32, grid_arr, norm, threads)


def diagnostics_sizes(w: dict):
    """Entries the diagnostics histograms need: (max support + 1, largest
    unclamped w-plane index of the points + 1), with the reference's float
    arithmetic."""
    p = place(w, single=True)
    return (int(np.max(w["support"])) + 1,
            int(p["raw_plane"].astype(np.int64).max(initial=0)) + 1)


def diagnostics_f(w: dict, use_reference: bool = False, init=None):
    """oskar_grid_wproj_f_diagnostics (restated, or the reference's own) on
    the arrays of `w`.  `init` optionally gives the starting contents of the
    in/out arrays (grid, norm, num_vis_per_wsupport, num_vis_per_wplane,
    num_vis_per_grid, avg_wsupport_per_grid, avg_wplane_per_grid); returns
    a dict of them and num_skipped."""
    a = _arrays(w, np.float32)
    g = w["grid_size"]
    ns, npl = diagnostics_sizes(w)
    out = dict(grid=np.zeros(2 * g * g, np.float32), norm=0.0,
               num_vis_per_wsupport=np.zeros(ns, np.int64),
               num_vis_per_wplane=np.zeros(npl, np.int64),
               num_vis_per_grid=np.zeros(g * g, np.int64),
               avg_wsupport_per_grid=np.zeros(g * g, np.float32),
               avg_wplane_per_grid=np.zeros(g * g, np.float32))
    if init:
        for k, v in init.items():
            out[k] = v if k == "norm" else np.array(v, copy=True)
    if use_reference:
        lib = reference_lib()
        if lib is None:
            raise RuntimeError("reference library not built")
        fn = lib.ref_oskar_grid_wproj_f_diagnostics
    else:
        fn = oracle_lib().orc_grid_wproj_f_diagnostics
    skipped = C.c_size_t(0)
    nrm = C.c_double(out["norm"])
    fn(w["num_w_planes"], _ptr(a["support"]), w["oversample"],
       w["conv_size_half"], _ptr(a["conv_func"]), a["uu"].shape[0],
       _ptr(a["uu"]), _ptr(a["vv"]), _ptr(a["ww"]), _ptr(a["vis"]),
       _ptr(a["weight"]), w["cell_size_rad"], w["w_scale"], g,
       C.byref(skipped), C.byref(nrm), _ptr(out["grid"]),
       _ptr(out["num_vis_per_wsupport"]), _ptr(out["num_vis_per_wplane"]),
       _ptr(out["num_vis_per_grid"]), _ptr(out["avg_wsupport_per_grid"]),
       _ptr(out["avg_wplane_per_grid"]))
    out["norm"] = nrm.value
    out["num_skipped"] = skipped.value
    return out


def place(w: dict, single: bool = False):
    """Per-visibility (gu, gv, plane, raw_plane, off_u, off_v, conj, skipped)
    with FP64 coordinates, or the reference _f's float ones if single."""
    lib = oracle_lib()
    dt = np.float32 if single else np.float64
    # placement needs only the coordinates and the support table
    a = {k: np.ascontiguousarray(w[k], dtype=dt) for k in ("uu", "vv", "ww")}
    a["support"] = np.ascontiguousarray(w["support"], dtype=np.int32)
    n = a["uu"].shape[0]
    outs = [np.zeros(n, np.int32) for _ in range(6)] + \
        [np.zeros(n, np.int8), np.zeros(n, np.uint8)]
    fn = lib.orc_vis_place_f if single else lib.orc_vis_place_d
    fn(w["num_w_planes"], _ptr(a["support"]), w["oversample"], n,
       _ptr(a["uu"]), _ptr(a["vv"]), _ptr(a["ww"]), w["cell_size_rad"],
       w["w_scale"], w["grid_size"], *[_ptr(o) for o in outs])
    keys = ("gu", "gv", "plane", "raw_plane", "off_u", "off_v", "conj",
            "skipped")
    return dict(zip(keys, outs))


def count_taps(w: dict) -> int:
    lib = oracle_lib()
    a = _arrays(w, np.float64)
    return int(lib.orc_count_taps_d(
        w["num_w_planes"], _ptr(a["support"]), w["oversample"],
        a["uu"].shape[0], _ptr(a["uu"]), _ptr(a["vv"]), _ptr(a["ww"]),
        w["cell_size_rad"], w["w_scale"], w["grid_size"]))


def time_parallel(w: dict, single: bool, threads: int, use_reference: bool,
                  want_grid: bool = False):
    """Time the reference's gridder (use_reference) or the restatement on
    `threads` threads with private grids.  The reference's FP32 function
    always processes exactly 10000 points (oskar_grid_wproj.c:155), so it is
    driven in consecutive 10000-point calls.  Returns
    (seconds, num_skipped, norm, grid or None)."""
    dt = np.float32 if single else np.float64
    a = _arrays(w, dt)
    g = w["grid_size"]
    out = np.zeros(2 * g * g, dtype=dt) if want_grid else None
    if use_reference:
        ref = reference_lib()
        if ref is None:
            raise RuntimeError("reference library not built (oracle/_ref)")
        fn = ref.ref_oskar_grid_wproj_f if single else ref.ref_oskar_grid_wproj_d
        chunk = 10000 if single else 0
    else:
        lib = oracle_lib()
        fn = lib.orc_grid_wproj_f if single else lib.orc_grid_wproj_d
        chunk = 0
    fnp = C.cast(fn, _P)
    skipped = C.c_size_t(0)
    nrm = C.c_double(0.0)
    timer = oracle_lib().orc_time_parallel_f if single else \
        oracle_lib().orc_time_parallel_d
    secs = timer(fnp, threads, chunk, w["num_w_planes"], _ptr(a["support"]),
                 w["oversample"], w["conv_size_half"], _ptr(a["conv_func"]),
                 a["uu"].shape[0], _ptr(a["uu"]), _ptr(a["vv"]),
                 _ptr(a["ww"]), _ptr(a["vis"]), _ptr(a["weight"]),
                 w["cell_size_rad"], w["w_scale"], g, C.byref(skipped),
                 C.byref(nrm), _ptr(out))
    if secs < 0:
        raise MemoryError("CPU baseline could not allocate private grids")
    return secs, skipped.value, nrm.value, out


def weights(uu, vv, weight, cell_size_rad, grid_size, grid, weight_out,
            single: bool = False, use_reference: bool = False):
    """Uniform weighting as the reference's main loop does it: the weights
    write (grid accumulates) then the read.  Arrays are copied, not
    modified.  Returns (skipped_write, grid, skipped_read, weight_out)."""
    sk_w, g, sk_r, wout, _ = weights_timed(uu, vv, weight, cell_size_rad,
                                           grid_size, grid, weight_out,
                                           single, use_reference)
    return sk_w, g, sk_r, wout


def weights_timed(uu, vv, weight, cell_size_rad, grid_size, grid, weight_out,
                  single: bool = False, use_reference: bool = False):
    """weights() that also returns the wall time of the write and read
    calls themselves (seconds, one host thread; the functions are serial):
    (skipped_write, grid, skipped_read, weight_out, (t_write, t_read))."""
    import time
    real = np.float32 if single else np.float64
    t = "f" if single else "d"
    lib = reference_lib() if use_reference else oracle_lib()
    prefix = "ref_oskar_" if use_reference else "orc_"
    a = [np.ascontiguousarray(x, dtype=real) for x in (uu, vv, weight)]
    g = np.array(grid, dtype=real, copy=True)
    wout = np.array(weight_out, dtype=real, copy=True)
    n = a[0].size
    sk_w = C.c_size_t(0)
    sk_r = C.c_size_t(0)
    cell = real(cell_size_rad)
    t0 = time.perf_counter()
    getattr(lib, prefix + "grid_weights_write_" + t)(
        n, _ptr(a[0]), _ptr(a[1]), _ptr(a[2]), cell, grid_size,
        C.byref(sk_w), _ptr(g))
    t1 = time.perf_counter()
    getattr(lib, prefix + "grid_weights_read_" + t)(
        n, _ptr(a[0]), _ptr(a[1]), _ptr(a[2]), _ptr(wout), cell, grid_size,
        C.byref(sk_r), _ptr(g))
    t2 = time.perf_counter()
    return sk_w.value, g, sk_r.value, wout, (t1 - t0, t2 - t1)


def time_weights_parallel(uu, vv, weight, cell_size_rad, grid_size,
                          threads: int, use_reference: bool):
    """FP32 uniform weighting on `threads` host threads: the reference's
    (use_reference) or the restated oskar_grid_weights_write_f on private
    grids over slices, a parallel sum of the grids, then _read_f over
    slices.  Returns (seconds, skipped_write, grid, skipped_read,
    weight_out); the grid equals the serial one whenever its sums are exact
    (e.g. unit weights)."""
    a = [np.ascontiguousarray(x, dtype=np.float32) for x in (uu, vv, weight)]
    n = a[0].size
    grid = np.zeros(grid_size * grid_size, np.float32)
    wout = np.zeros(n, np.float32)
    if use_reference:
        lib = reference_lib()
        if lib is None:
            raise RuntimeError("reference library not built (oracle/_ref)")
        prefix = "ref_oskar_"
    else:
        lib = oracle_lib()
        prefix = "orc_"
    wfn = C.cast(getattr(lib, prefix + "grid_weights_write_f"), _P)
    rfn = C.cast(getattr(lib, prefix + "grid_weights_read_f"), _P)
    sk_w = C.c_size_t(0)
    sk_r = C.c_size_t(0)
    secs = oracle_lib().orc_time_weights_parallel_f(
        wfn, rfn, threads, n, _ptr(a[0]), _ptr(a[1]), _ptr(a[2]),
        np.float32(cell_size_rad), grid_size, _ptr(grid), _ptr(wout),
        C.byref(sk_w), C.byref(sk_r))
    if secs < 0:
        raise MemoryError("CPU baseline could not allocate private grids")
    return secs, sk_w.value, grid, sk_r.value, wout


def degrid_d(w: dict, grid_arr, vis_out=None):
    """The adjoint of the gridder (orc_degrid_wproj_d) on the arrays of `w`
    (FP64) and a complex FP64 grid.  Returns (num_skipped, vis_out)."""
    a = _arrays(w, np.float64)
    n = a["uu"].shape[0]
    out = np.zeros(2 * n) if vis_out is None else \
        np.array(vis_out, dtype=np.float64, copy=True)
    g = np.ascontiguousarray(grid_arr, dtype=np.float64)
    sk = C.c_size_t(0)
    oracle_lib().orc_degrid_wproj_d(
        w["num_w_planes"], _ptr(a["support"]), w["oversample"],
        w["conv_size_half"], _ptr(a["conv_func"]), n, _ptr(a["uu"]),
        _ptr(a["vv"]), _ptr(a["ww"]), w["cell_size_rad"], w["w_scale"],
        w["grid_size"], _ptr(g), C.byref(sk), _ptr(out))
    return sk.value, out


def rel_rms(test: np.ndarray, ref: np.ndarray) -> float:
    """The reference harness's grid error metric (main.cpp:575-598):
    sqrt(sum |test - ref|^2) / sqrt(sum |ref|^2), accumulated in FP64."""
    t = np.asarray(test, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    den = np.sqrt(np.sum(r * r))
    num = np.sqrt(np.sum((t - r) ** 2))
    return float(num / den) if den > 0 else float(num)
