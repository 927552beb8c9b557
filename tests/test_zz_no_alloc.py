"""oskar_b200_grid_f_static: gridding for callers that cannot allocate
device memory (a fixed memory pool, memory provisioned up front by a
scheduler, or a thread that must not take the allocator's locks while other
streams run).  Its scratch is one static device array shared by every call,
so this file runs last: two calls in a row through the C ABI must match the
allocating entry point (oskar_b200_grid) within the FP32 tolerance, and a
job larger than the static scratch must be refused before any device work.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import fpga_gridding_b200 as fg
from fpga_gridding_b200 import _lib, workloads as W
from oracle.oracle import rel_rms

pytestmark = pytest.mark.gpu

TOL_F = 1e-5


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


@pytest.fixture(scope="module")
def job():
    w = W.plain_small().to(dtype=torch.float32)
    d = dict(wl=w, uu=w.uu.cuda(), vv=w.vv.cuda(), ww=w.ww.cuda(),
             vis=w.vis.cuda(), weight=w.weight.cuda(),
             cube=w.conv_func.float().cuda(),
             support=np.ascontiguousarray(w.support, np.int32),
             cell=float(np.float32(w.cell_size_rad)),
             wsc=float(np.float32(w.w_scale)), g=w.grid_size)
    return d


def _static_call(lib, j, grid, skip, norm, n=None):
    return lib.oskar_b200_grid_f_static(
        len(j["support"]), j["support"].ctypes.data_as(C.c_void_p),
        j["wl"].oversample, j["wl"].conv_size_half, _ptr(j["cube"]),
        j["uu"].numel() if n is None else n, _ptr(j["uu"]), _ptr(j["vv"]),
        _ptr(j["ww"]), _ptr(j["vis"]), j["cell"], j["wsc"], j["g"],
        _ptr(grid), _ptr(skip), _ptr(norm), None)


def test_static_entry_matches_allocating_entry_twice(job):
    lib = fg.load()
    g = job["g"]
    # the existing, allocating entry point
    ws = fg.Workspace(0)
    cube = fg.Cube(ws, job["support"], job["wl"].oversample,
                   job["wl"].conv_size_half, job["cube"],
                   data_is_double=False)
    ref = torch.zeros(2 * g * g, device="cuda")
    rskip = torch.zeros(1, dtype=torch.int64, device="cuda")
    rnorm = torch.zeros(1, dtype=torch.float64, device="cuda")
    fg.grid_device(ws, cube, job["uu"], job["vv"], job["ww"], job["vis"],
                   job["weight"], job["cell"], job["wsc"], g, ref, rskip,
                   rnorm)
    torch.cuda.synchronize()
    ref_np = ref.cpu().numpy()
    for _ in range(2):
        grid = torch.zeros(2 * g * g, device="cuda")
        skip = torch.full((1,), 12345, dtype=torch.int64, device="cuda")
        norm = torch.zeros(1, dtype=torch.float64, device="cuda")
        assert _static_call(lib, job, grid, skip, norm) == _lib.OK
        torch.cuda.synchronize()
        assert int(skip.item()) == int(rskip.item())
        assert abs(norm.item() - rnorm.item()) <= 1e-12 * abs(rnorm.item())
        assert rel_rms(grid.cpu().numpy(), ref_np) <= TOL_F
    cube.close()
    ws.close()


def test_static_entry_refuses_jobs_beyond_its_scratch(job):
    lib = fg.load()
    grid = torch.zeros(2 * job["g"] ** 2, device="cuda")
    skip = torch.zeros(1, dtype=torch.int64, device="cuda")
    norm = torch.zeros(1, dtype=torch.float64, device="cuda")
    # 4 million points need ~290 MB of scratch: refused before any device
    # work (the pointers are never read)
    st = _static_call(lib, job, grid, skip, norm, n=4_000_000)
    assert st == _lib.ERR_OVER_BUDGET
    torch.cuda.synchronize()
    assert not grid.any() and int(skip.item()) == 0 and norm.item() == 0.0
