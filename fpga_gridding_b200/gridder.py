"""Python front end of the B200 gridder.

`oskar_grid_wproj_d` / `oskar_grid_wproj_f` mirror the reference's C
functions (oskar_grid_wproj.h:69-86, :114-131): same argument order and
meaning, host (numpy) arrays, grid updated in place.  The C out-parameters
num_skipped and norm come back as the return value (num_skipped, norm),
norm being the updated accumulator.  Failures raise GridderError instead of
the reference's silent behaviour.

`Workspace`, `Cube`, `grid_device` and `place_device` wrap the extended,
device-resident API for torch CUDA tensors.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import GridderError, Options, Stats, check, load


def _carr(a, dtype):
    a = np.asarray(a)
    if a.dtype != dtype or not a.flags.c_contiguous:
        raise TypeError(f"expected a C-contiguous {np.dtype(dtype).name} array")
    return a.ctypes.data_as(C.c_void_p)


def _dropin(fn, real, num_w_planes, support, oversample, conv_size_half,
            conv_func, num_points, uu, vv, ww, vis, weight, cell_size_rad,
            w_scale, grid_size, norm, grid):
    lib = load()
    support = np.ascontiguousarray(support, dtype=np.int32)
    skipped = C.c_size_t(0)
    nrm = C.c_double(norm)
    args = [num_w_planes, _carr(support, np.int32), oversample,
            conv_size_half, _carr(conv_func, real), num_points]
    for a in (uu, vv, ww, vis):
        args.append(_carr(a, real))
    args.append(_carr(weight, real) if weight is not None else None)
    args += [cell_size_rad, w_scale, grid_size, C.byref(skipped),
             C.byref(nrm), _carr(grid, real)]
    fn(*args)
    check(lib.oskar_grid_wproj_b200_last_error(), fn.__name__)
    return skipped.value, nrm.value


def oskar_grid_wproj_d(num_w_planes, support, oversample, conv_size_half,
                       conv_func, num_points, uu, vv, ww, vis, weight,
                       cell_size_rad, w_scale, grid_size, norm, grid):
    """FP64 drop-in.  Returns (num_skipped, norm); grid accumulates."""
    return _dropin(load().oskar_grid_wproj_d, np.float64, num_w_planes,
                   support, oversample, conv_size_half, conv_func,
                   num_points, uu, vv, ww, vis, weight, cell_size_rad,
                   w_scale, grid_size, norm, grid)


def oskar_grid_wproj_f(num_w_planes, support, oversample, conv_size_half,
                       conv_func, num_points, uu, vv, ww, vis, weight,
                       cell_size_rad, w_scale, grid_size, norm, grid):
    """FP32 drop-in (FP64 coordinates).  Returns (num_skipped, norm)."""
    return _dropin(load().oskar_grid_wproj_f, np.float32, num_w_planes,
                   support, oversample, conv_size_half, conv_func,
                   num_points, uu, vv, ww, vis, weight, cell_size_rad,
                   w_scale, grid_size, norm, grid)


def oskar_grid_wproj_f_diagnostics(num_w_planes, support, oversample,
                                   conv_size_half, conv_func, num_points, uu,
                                   vv, ww, vis, weight, cell_size_rad,
                                   w_scale, grid_size, norm, grid,
                                   num_vis_per_wsupport, num_vis_per_wplane,
                                   num_vis_per_grid, avg_wsupport_per_grid,
                                   avg_wplane_per_grid):
    """oskar_grid_wproj.c:245-370 on the GPU: the float-coordinate FP32
    gridder plus hit counts.  The grid (float32), the int64 count arrays and
    avg_wsupport_per_grid (float32) accumulate in place; returns
    (num_skipped, norm)."""
    lib = load()
    support = np.ascontiguousarray(support, dtype=np.int32)
    # The library writes as many entries as the reference's indexing needs;
    # refuse arrays too small for them instead of letting it write past
    # their ends.  The largest plane index in the float arithmetic:
    # roundf(sqrtf(|w * w_scale|)), half away from zero.
    # (Indices that are not finite or not below 2^24 make the library refuse
    # the call before it writes anything.)
    cells = grid_size * grid_size
    plane_max = -1
    if num_points:
        r = np.sqrt(np.abs(np.asarray(ww, np.float32)[:num_points] *
                           np.float32(w_scale)))
        top = np.floor(r.astype(np.float64) + 0.5).max()
        if np.isfinite(top) and top < 2 ** 24:
            plane_max = int(top)
    for arr, need, name in (
            (num_vis_per_wsupport, int(support.max()) + 1,
             "num_vis_per_wsupport"),
            (num_vis_per_wplane, plane_max + 1, "num_vis_per_wplane"),
            (num_vis_per_grid, cells, "num_vis_per_grid"),
            (avg_wsupport_per_grid, cells, "avg_wsupport_per_grid")):
        if np.asarray(arr).size < need:
            raise ValueError(f"{name} holds {np.asarray(arr).size} entries; "
                             f"this call needs {need}")
    skipped = C.c_size_t(0)
    nrm = C.c_double(norm)
    fn = lib.oskar_grid_wproj_f_diagnostics
    fn(num_w_planes, _carr(support, np.int32), oversample, conv_size_half,
       _carr(conv_func, np.float32), num_points, _carr(uu, np.float32),
       _carr(vv, np.float32), _carr(ww, np.float32), _carr(vis, np.float32),
       _carr(weight, np.float32) if weight is not None else None,
       cell_size_rad, w_scale, grid_size, C.byref(skipped), C.byref(nrm),
       _carr(grid, np.float32), _carr(num_vis_per_wsupport, np.int64),
       _carr(num_vis_per_wplane, np.int64), _carr(num_vis_per_grid, np.int64),
       _carr(avg_wsupport_per_grid, np.float32),
       _carr(avg_wplane_per_grid, np.float32)
       if avg_wplane_per_grid is not None else None)
    check(lib.oskar_grid_wproj_b200_last_error(), fn.__name__)
    return skipped.value, nrm.value


def grid_workload(w: dict, single: bool, grid=None, norm: float = 0.0):
    """Drop-in call on a Workload.numpy() dict.  Returns
    (num_skipped, norm, grid)."""
    real = np.float32 if single else np.float64
    g = w["grid_size"]
    if grid is None:
        grid = np.zeros(2 * g * g, dtype=real)
    fn = oskar_grid_wproj_f if single else oskar_grid_wproj_d
    conv = lambda k: np.ascontiguousarray(w[k], dtype=real)
    sk, nrm = fn(w["num_w_planes"], w["support"], w["oversample"],
                 w["conv_size_half"], conv("conv_func"), len(w["uu"]),
                 conv("uu"), conv("vv"), conv("ww"), conv("vis"),
                 conv("weight"), w["cell_size_rad"], w["w_scale"], g, norm,
                 grid)
    return sk, nrm, grid


def _weights_write(t, real, num_points, uu, vv, weight, cell_size_rad,
                   grid_size, grid):
    lib = load()
    fn = getattr(lib, "oskar_grid_weights_write_" + t)
    skipped = C.c_size_t(0)
    fn(num_points, _carr(uu, real), _carr(vv, real), _carr(weight, real),
       cell_size_rad, grid_size, C.byref(skipped), _carr(grid, real))
    check(lib.oskar_grid_wproj_b200_last_error(), fn.__name__)
    return skipped.value


def _weights_read(t, real, num_points, uu, vv, weight_in, weight_out,
                  cell_size_rad, grid_size, grid):
    lib = load()
    fn = getattr(lib, "oskar_grid_weights_read_" + t)
    skipped = C.c_size_t(0)
    fn(num_points, _carr(uu, real), _carr(vv, real), _carr(weight_in, real),
       _carr(weight_out, real), cell_size_rad, grid_size, C.byref(skipped),
       _carr(grid, real))
    check(lib.oskar_grid_wproj_b200_last_error(), fn.__name__)
    return skipped.value


def oskar_grid_weights_write_d(num_points, uu, vv, weight, cell_size_rad,
                               grid_size, grid):
    """utils/oskar_grid_weights.c:38-69 on the GPU.  grid (grid_size^2
    float64) accumulates in place; returns num_skipped."""
    return _weights_write("d", np.float64, num_points, uu, vv, weight,
                          cell_size_rad, grid_size, grid)


def oskar_grid_weights_read_d(num_points, uu, vv, weight_in, weight_out,
                              cell_size_rad, grid_size, grid):
    """utils/oskar_grid_weights.c:71-103 on the GPU.  weight_out is updated
    in place; returns num_skipped."""
    return _weights_read("d", np.float64, num_points, uu, vv, weight_in,
                         weight_out, cell_size_rad, grid_size, grid)


def oskar_grid_weights_write_f(num_points, uu, vv, weight, cell_size_rad,
                               grid_size, grid):
    """utils/oskar_grid_weights.c:105-136 (float) on the GPU."""
    return _weights_write("f", np.float32, num_points, uu, vv, weight,
                          cell_size_rad, grid_size, grid)


def oskar_grid_weights_read_f(num_points, uu, vv, weight_in, weight_out,
                              cell_size_rad, grid_size, grid):
    """utils/oskar_grid_weights.c:138-170 (float) on the GPU."""
    return _weights_read("f", np.float32, num_points, uu, vv, weight_in,
                         weight_out, cell_size_rad, grid_size, grid)


# --------------------------------------------------------------------------
# Extended API (device-resident, torch tensors)
# --------------------------------------------------------------------------

def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream_ptr(stream):
    if stream is None:
        return None
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream")
                      else int(stream))


def options(**kw) -> Options:
    o = Options()
    load().oskar_b200_options_init(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Workspace:
    """Device buffers and a default stream for one device."""

    def __init__(self, device: int = 0):
        self._lib = load()
        self.handle = C.c_void_p()
        check(self._lib.oskar_b200_workspace_create(device,
                                                   C.byref(self.handle)),
              "workspace_create")
        self.device = device

    def close(self):
        if self.handle:
            self._lib.oskar_b200_workspace_free(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def bytes(self) -> int:
        return int(self._lib.oskar_b200_workspace_bytes(self.handle))

    def autotune(self, cube, uu, vv, ww, vis, cell_size_rad: float,
                 w_scale: float, grid_size: int, grid,
                 opts: Options | None = None) -> np.ndarray:
        """Measures the fastest classes-per-thread per support, then the
        tile width and kernel-value path, and (with compensated accumulation
        in `opts`) the compensation radius on a sample job (device tensors;
        `grid` is scratch), and keeps them for later calls on this
        workspace.  Returns the classes-per-thread table (index = support);
        tune_launch() reads the rest."""
        table = np.zeros(128, np.uint8)
        check(self._lib.oskar_b200_autotune(
            self.handle, cube.handle,
            C.byref(opts) if opts is not None else None, uu.numel(),
            _ptr(uu), _ptr(vv), _ptr(ww), _ptr(vis), float(cell_size_rad),
            float(w_scale), grid_size, _ptr(grid),
            table.ctypes.data_as(C.c_void_p)), "autotune")
        return table

    def tune_table(self, table=None) -> np.ndarray:
        """Sets the classes-per-thread table (128 entries) if given; returns
        the table in use."""
        cur = np.zeros(128, np.uint8)
        t = None
        if table is not None:
            t = np.ascontiguousarray(table, dtype=np.uint8)
        check(self._lib.oskar_b200_tune_table(
            self.handle, t.ctypes.data_as(C.c_void_p) if t is not None
            else None, cur.ctypes.data_as(C.c_void_p)), "tune_table")
        return cur

    def tune_launch(self, shape=None) -> tuple:
        """Sets the launch shape (tile_shift, staging, compensate_radius)
        that calls leaving these to the workspace use, if given; returns the
        shape in use."""
        cur = (C.c_int * 3)()
        arr = None
        if shape is not None:
            arr = (C.c_int * 3)(*[int(x) for x in shape])
        check(self._lib.oskar_b200_tune_launch(
            self.handle, arr, cur), "tune_launch")
        return tuple(cur)

    def stats(self) -> Stats:
        s = Stats()
        check(self._lib.oskar_b200_last_stats(self.handle, C.byref(s)),
              "last_stats")
        return s


class Cube:
    """A W-kernel cube re-laid and resident on the device."""

    def __init__(self, ws: Workspace, support, oversample: int,
                 conv_size_half: int, conv_func, data_is_double: bool,
                 kernel_type: int = _lib.KERNEL_NATIVE, stream=None,
                 conv_imag=None):
        """conv_func: the interleaved complex cube (reference layout), or,
        with conv_imag given, its real part (the two cubes read_kernel
        returns).  numpy arrays (host) or CUDA tensors (device)."""
        import torch
        self._lib = load()
        self.support = np.ascontiguousarray(support, dtype=np.int32)
        on_device = isinstance(conv_func, torch.Tensor) and conv_func.is_cuda

        def ref(a):
            if isinstance(a, torch.Tensor):
                a = a.contiguous()
                return a, a.dtype == torch.float64, C.c_void_p(a.data_ptr())
            a = np.ascontiguousarray(a)
            return a, a.dtype == np.float64, a.ctypes.data_as(C.c_void_p)
        conv_func, is_double, ptr = ref(conv_func)
        self._keep = [conv_func]
        self.handle = C.c_void_p()
        sup = self.support.ctypes.data_as(C.c_void_p)
        if conv_imag is None:
            check(self._lib.oskar_b200_cube_create(
                ws.handle, len(self.support), sup, oversample,
                conv_size_half, ptr, int(is_double), int(on_device),
                int(data_is_double), kernel_type, _stream_ptr(stream),
                C.byref(self.handle)), "cube_create")
        else:
            conv_imag, im_double, im_ptr = ref(conv_imag)
            if im_double != is_double:
                raise TypeError("real and imaginary cubes differ in dtype")
            self._keep.append(conv_imag)
            check(self._lib.oskar_b200_cube_create_planar(
                ws.handle, len(self.support), sup, oversample,
                conv_size_half, ptr, im_ptr, int(is_double), int(on_device),
                int(data_is_double), kernel_type, _stream_ptr(stream),
                C.byref(self.handle)), "cube_create_planar")
        self._keep = None   # the constructor is synchronous
        self.data_is_double = data_is_double
        self.kernel_type = kernel_type

    def close(self):
        if self.handle:
            self._lib.oskar_b200_cube_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def bytes(self) -> int:
        return int(self._lib.oskar_b200_cube_bytes(self.handle))


def grid_device(ws: Workspace, cube: Cube, uu, vv, ww, vis, weight,
                cell_size_rad: float, w_scale: float, grid_size: int, grid,
                d_num_skipped=None, d_norm=None, opts: Options | None = None,
                stream=None) -> None:
    """Asynchronous gridding of device tensors into `grid` (accumulates).
    d_num_skipped (uint64/int64 device scalar) is overwritten, d_norm
    (float64 device scalar) incremented."""
    lib = load()
    if opts is None:
        opts = options()
    n = uu.numel()
    check(lib.oskar_b200_grid(
        ws.handle, cube.handle, C.byref(opts), n, _ptr(uu), _ptr(vv),
        _ptr(ww), _ptr(vis), _ptr(weight), float(cell_size_rad),
        float(w_scale), grid_size, _ptr(grid), _ptr(d_num_skipped),
        _ptr(d_norm), _stream_ptr(stream)), "oskar_b200_grid")


def degrid_device(ws: Workspace, cube: Cube, uu, vv, ww, weight,
                  cell_size_rad: float, w_scale: float, grid_size: int, grid,
                  vis, d_num_skipped=None, opts: Options | None = None,
                  stream=None) -> None:
    """Asynchronous degridding (the adjoint of grid_device): reads the
    device `grid`, writes the kept visibilities' values into `vis`."""
    lib = load()
    if opts is None:
        opts = options()
    check(lib.oskar_b200_degrid(
        ws.handle, cube.handle, C.byref(opts), uu.numel(), _ptr(uu),
        _ptr(vv), _ptr(ww), _ptr(weight), float(cell_size_rad),
        float(w_scale), grid_size, _ptr(grid), _ptr(vis),
        _ptr(d_num_skipped), _stream_ptr(stream)), "oskar_b200_degrid")


def degrid_host(ws: Workspace, cube: Cube, uu, vv, ww, weight,
                cell_size_rad: float, w_scale: float, grid_size: int, grid,
                vis, opts: Options | None = None) -> int:
    """Synchronous degridding of host numpy arrays (float32 for an FP32
    cube, float64 for FP64): `grid` is read, the kept visibilities' values
    are written into `vis` (interleaved complex).  Returns the skip count.
    The copies overlap the work (oskar_b200_degrid_host)."""
    lib = load()
    if opts is None:
        opts = options()
    real = np.float64 if cube.data_is_double else np.float32
    for name, a in (("uu", uu), ("vv", vv), ("ww", ww), ("grid", grid),
                    ("vis", vis)):
        if not (isinstance(a, np.ndarray) and a.dtype == real and
                a.flags["C_CONTIGUOUS"]):
            raise TypeError(f"{name} must be a contiguous {real.__name__} "
                            "numpy array")
    w = None
    if opts.apply_weight:
        w = np.ascontiguousarray(weight, dtype=real)
    skipped = C.c_size_t(0)
    check(lib.oskar_b200_degrid_host(
        ws.handle, cube.handle, C.byref(opts), uu.size, uu.ctypes.data,
        vv.ctypes.data, ww.ctypes.data,
        w.ctypes.data if w is not None else None, float(cell_size_rad),
        float(w_scale), grid_size, grid.ctypes.data, vis.ctypes.data,
        C.byref(skipped)), "oskar_b200_degrid_host")
    return skipped.value


def grid_batch_device(ws: Workspace, jobs, opts: Options | None = None,
                      stream=None) -> None:
    """Asynchronous batched gridding.  `jobs` is a sequence of dicts with
    the keys of grid_device: cube, uu, vv, ww, vis, weight, cell_size_rad,
    w_scale, grid_size, grid and optionally d_num_skipped, d_norm (device
    tensors).  One sort and one persistent gridding launch serve all jobs."""
    lib = load()
    if opts is None:
        opts = options()
    arr = (_lib.Job * len(jobs))()
    keep = []
    for i, j in enumerate(jobs):
        arr[i].cube = j["cube"].handle
        arr[i].num_points = j["uu"].numel()
        for k in ("uu", "vv", "ww", "vis", "weight", "grid", "d_num_skipped",
                  "d_norm"):
            t = j.get(k)
            setattr(arr[i], k, t.data_ptr() if t is not None else None)
            keep.append(t)
        arr[i].cell_size_rad = float(j["cell_size_rad"])
        arr[i].w_scale = float(j["w_scale"])
        arr[i].grid_size = int(j["grid_size"])
        arr[i].frequency_hz = float(j.get("frequency_hz", 0.0))
    check(lib.oskar_b200_grid_batch(ws.handle, C.byref(opts), len(jobs), arr,
                                    _stream_ptr(stream)),
          "oskar_b200_grid_batch")


def place_device(ws: Workspace, support, oversample: int, uu, vv, ww,
                 cell_size_rad: float, w_scale: float, grid_size: int,
                 coord_mode: int = _lib.COORDS_F64, stream=None) -> dict:
    """Per-visibility placement as computed on the device (synchronous).
    Returns int32 device tensors gu, gv, plane, off_u, off_v, conj, skipped."""
    import torch
    lib = load()
    support = np.ascontiguousarray(support, dtype=np.int32)
    n = uu.numel()
    out = {k: torch.empty(n, dtype=torch.int32, device=uu.device)
           for k in ("gu", "gv", "plane", "off_u", "off_v", "conj", "skipped")}
    check(lib.oskar_b200_place(
        ws.handle, int(uu.dtype == torch.float64), coord_mode, len(support),
        support.ctypes.data_as(C.c_void_p), oversample, n, _ptr(uu),
        _ptr(vv), _ptr(ww), float(cell_size_rad), float(w_scale), grid_size,
        *[_ptr(out[k]) for k in ("gu", "gv", "plane", "off_u", "off_v",
                                 "conj", "skipped")],
        _stream_ptr(stream)), "oskar_b200_place")
    return out


def weights_write_device(ws: Workspace, uu, vv, weight, cell_size_rad,
                         grid_size: int, grid, num_skipped=None,
                         ordered: bool = True, frequency_hz: float = 0.0,
                         stream=None):
    """Weights-grid histogram on torch CUDA tensors (float32 or float64);
    grid (grid_size^2 reals) accumulates.  ordered=True is bit-identical to
    the reference; ordered=False uses one atomic add per point.
    frequency_hz > 0: uu, vv are in metres (scaled as scale_coords does)."""
    dbl = uu.dtype.is_floating_point and uu.element_size() == 8
    check(ws._lib.oskar_b200_weights_write(
        ws.handle, int(dbl), int(ordered), uu.numel(), _ptr(uu), _ptr(vv),
        _ptr(weight), float(cell_size_rad), grid_size, _ptr(grid),
        _ptr(num_skipped), float(frequency_hz), _stream_ptr(stream)),
        "weights_write")


def weights_read_device(ws: Workspace, uu, vv, weight_in, weight_out,
                        cell_size_rad, grid_size: int, grid,
                        num_skipped=None, frequency_hz: float = 0.0,
                        stream=None):
    """Density lookup on torch CUDA tensors: weight_out = weight_in /
    grid[cell] (0 for empty cells; skipped points keep weight_out)."""
    dbl = uu.element_size() == 8
    check(ws._lib.oskar_b200_weights_read(
        ws.handle, int(dbl), uu.numel(), _ptr(uu), _ptr(vv), _ptr(weight_in),
        _ptr(weight_out), float(cell_size_rad), grid_size, _ptr(grid),
        _ptr(num_skipped), float(frequency_hz), _stream_ptr(stream)),
        "weights_read")


class Blocks:
    """Block ingest (oskar_b200_blocks_*): host visibility blocks streamed
    into one device grid.  push() takes host numpy arrays (the cube's
    precision) and returns once they have been copied; the block grids
    while the caller prepares the next.  finish() waits and returns the
    total number of skipped points."""

    def __init__(self, ws: Workspace, cube: Cube, cell_size_rad: float,
                 w_scale: float, grid_size: int, grid, d_norm=None,
                 opts: Options | None = None):
        self._lib = load()
        self._keep = (ws, cube, grid, d_norm)
        self.handle = C.c_void_p()
        check(self._lib.oskar_b200_blocks_create(
            ws.handle, cube.handle, C.byref(opts) if opts is not None else None,
            float(cell_size_rad), float(w_scale), grid_size, _ptr(grid),
            _ptr(d_norm), C.byref(self.handle)), "blocks_create")
        self._real = np.float64 if cube.data_is_double else np.float32

    def push(self, uu, vv, ww, vis, weight=None, frequency_hz: float = 0.0):
        r = self._real
        arrs = [np.ascontiguousarray(a, dtype=r) for a in (uu, vv, ww, vis)]
        w = np.ascontiguousarray(weight, dtype=r) if weight is not None \
            else None
        check(self._lib.oskar_b200_blocks_push(
            self.handle, arrs[0].size, *[a.ctypes.data_as(C.c_void_p)
                                         for a in arrs],
            w.ctypes.data_as(C.c_void_p) if w is not None else None,
            float(frequency_hz)), "blocks_push")

    def finish(self) -> int:
        sk = C.c_ulonglong(0)
        check(self._lib.oskar_b200_blocks_finish(self.handle, C.byref(sk)),
              "blocks_finish")
        return sk.value

    def close(self):
        if self.handle:
            self._lib.oskar_b200_blocks_free(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
