"""Python front end of the resident gridding server (oskar_b200_server_*).

The server runs in the library's own thread: it admits submitted jobs as
slots and HBM budget free up, merges queued jobs into batched launches, runs
slots concurrently on their own streams, and reports per-job submit / start
/ end times on its clock.  Job inputs and cubes are the caller's device
memory and must stay alive until the job completes; each result grid is the
server's until released.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import Completion, Request, check, load


class _DeviceArray:
    """A raw device pointer seen by torch (no ownership)."""

    def __init__(self, ptr, n, dtype):
        typestr = {torch.float32: "<f4", torch.float64: "<f8"}[dtype]
        self.__cuda_array_interface__ = {
            "shape": (n,), "typestr": typestr, "data": (ptr, False),
            "version": 3, "strides": None}


class Server:
    def __init__(self, device: int = 0, budget_bytes: int = 150 << 30,
                 slots: int = 4, max_batch: int = 32, opts=None):
        self._lib = load()
        self.handle = C.c_void_p()
        o = opts if opts is not None else _lib.Options()
        if opts is None:
            self._lib.oskar_b200_options_init(C.byref(o))
        check(self._lib.oskar_b200_server_create(
            device, int(budget_bytes), slots, max_batch, C.byref(o),
            C.byref(self.handle)), "server_create")
        self._inflight = {}   # tag -> tensors kept alive until completion
        self._meta = {}       # tag -> (grid_size, dtype)

    def submit(self, tag: int, cube, uu, vv, ww, vis, weight,
               cell_size_rad: float, w_scale: float, grid_size: int,
               frequency_hz: float = 0.0) -> None:
        r = Request()
        r.tag = tag
        r.cube = cube.handle
        r.num_points = uu.numel()
        r.uu, r.vv, r.ww, r.vis = (t.data_ptr() for t in (uu, vv, ww, vis))
        r.weight = weight.data_ptr() if weight is not None else None
        r.cell_size_rad = float(cell_size_rad)
        r.w_scale = float(w_scale)
        r.grid_size = int(grid_size)
        r.frequency_hz = float(frequency_hz)
        self._inflight[tag] = (uu, vv, ww, vis, weight, cube)
        self._meta[tag] = (grid_size, uu.dtype)
        check(self._lib.oskar_b200_server_submit(self.handle, C.byref(r)),
              "server_submit")

    def poll(self, max_out: int = 256, timeout: float = 0.05) -> list:
        buf = (Completion * max_out)()
        n = C.c_int(0)
        check(self._lib.oskar_b200_server_poll(self.handle, buf, max_out,
                                               C.byref(n), float(timeout)),
              "server_poll")
        out = []
        for i in range(n.value):
            c = buf[i]
            self._inflight.pop(c.tag, None)
            out.append(dict(tag=c.tag, status=c.status,
                            num_skipped=c.num_skipped, norm=c.norm,
                            grid_ptr=c.grid, submit_s=c.submit_s,
                            start_s=c.start_s, end_s=c.end_s,
                            batch_size=c.batch_size))
        return out

    def grid(self, completion) -> torch.Tensor:
        """The completed job's grid as a torch view (valid until release)."""
        g, dtype = self._meta[completion["tag"]]
        arr = _DeviceArray(completion["grid_ptr"], 2 * g * g, dtype)
        return torch.as_tensor(arr, device="cuda")

    def release(self, tag: int) -> None:
        self._meta.pop(tag, None)
        check(self._lib.oskar_b200_server_release(self.handle, tag),
              "server_release")

    def clock(self) -> float:
        return float(self._lib.oskar_b200_server_clock(self.handle))

    def memory(self):
        used, budget = C.c_size_t(0), C.c_size_t(0)
        check(self._lib.oskar_b200_server_memory(self.handle, C.byref(used),
                                                 C.byref(budget)),
              "server_memory")
        return used.value, budget.value

    def close(self) -> None:
        if self.handle:
            self._lib.oskar_b200_server_free(self.handle)
            self.handle = C.c_void_p()
            self._inflight.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
