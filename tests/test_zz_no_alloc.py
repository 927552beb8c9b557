"""oskar_b200_grid_f_static: gridding for callers that cannot allocate
device memory (a fixed memory pool, memory provisioned up front by a
scheduler, or a thread that must not take the allocator's locks while other
streams run).  Its scratch is one static device array shared by every call,
so this file runs last: two calls in a row through the C ABI must match the
allocating entry point (oskar_b200_grid) within the FP32 tolerance, a job
larger than the static scratch must be refused before any device work, and
the device status word that the kernels' checks write into the array must be
readable (oskar_b200_grid_f_static_status) and cleared by every call.
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


def _job(w):
    return dict(wl=w, uu=w.uu.cuda(), vv=w.vv.cuda(), ww=w.ww.cuda(),
                vis=w.vis.cuda(), weight=w.weight.cuda(),
                cube=w.conv_func.float().cuda(),
                support=np.ascontiguousarray(w.support, np.int32),
                cell=float(np.float32(w.cell_size_rad)),
                wsc=float(np.float32(w.w_scale)), g=w.grid_size)


def _static_status(lib):
    st = C.c_int(-1)
    assert lib.oskar_b200_grid_f_static_status(None, C.byref(st)) == _lib.OK
    return st.value


def _allocating(j, n=None):
    """The allocating entry point's grid, skip count and norm."""
    g = j["g"]
    ws = fg.Workspace(0)
    cube = fg.Cube(ws, j["support"], j["wl"].oversample,
                   j["wl"].conv_size_half, j["cube"], data_is_double=False)
    sl = slice(0, j["uu"].numel() if n is None else n)
    ref = torch.zeros(2 * g * g, device="cuda")
    rskip = torch.zeros(1, dtype=torch.int64, device="cuda")
    rnorm = torch.zeros(1, dtype=torch.float64, device="cuda")
    fg.grid_device(ws, cube, j["uu"][sl], j["vv"][sl], j["ww"][sl],
                   j["vis"][2 * sl.start:2 * sl.stop], j["weight"][sl],
                   j["cell"], j["wsc"], g, ref, rskip, rnorm)
    torch.cuda.synchronize()
    out = (ref.cpu().numpy(), int(rskip.item()), float(rnorm.item()))
    cube.close()
    ws.close()
    return out


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
    # 4 million points need ~165 MB of scratch: refused before any device
    # work (the pointers are never read)
    st = _static_call(lib, job, grid, skip, norm, n=4_000_000)
    assert st == _lib.ERR_OVER_BUDGET
    torch.cuda.synchronize()
    assert not grid.any() and int(skip.item()) == 0 and norm.item() == 0.0


def test_static_status_reads_ok_after_a_normal_call(job):
    lib = fg.load()
    g = job["g"]
    grid = torch.zeros(2 * g * g, device="cuda")
    assert _static_call(lib, job, grid, None, None) == _lib.OK
    assert _static_status(lib) == _lib.OK


def test_static_status_reports_planted_bits_and_each_call_clears_them(job):
    """The bits a kernel's bounds check or bounded wait would set are planted
    on the host side (no fault is provoked on the GPU); the reader maps them
    to the library's status codes, and the next gridding call starts from a
    clear word."""
    lib = fg.load()
    g = job["g"]
    grid = torch.zeros(2 * g * g, device="cuda")
    for bits, want in ((1, _lib.ERR_DEVICE_CHECK), (8, _lib.ERR_DEVICE_CHECK),
                       (4, _lib.ERR_TIMEOUT), (5, _lib.ERR_TIMEOUT)):
        assert lib.oskar_b200_testing_set_static_status(bits, None) == _lib.OK
        assert _static_status(lib) == want
        assert _static_call(lib, job, grid, None, None) == _lib.OK
        assert _static_status(lib) == _lib.OK


def test_static_entry_on_a_second_workload_and_without_outputs():
    """A job with other supports, plane count and grid size after the first
    one (stale slabs, norm table or histograms of the previous call would
    show), then the same job with NULL skip and norm pointers, then an empty
    job: each against the allocating entry point."""
    lib = fg.load()
    w = W.plain_small(seed=7, num_stations=20, num_times=30, grid_size=512,
                      num_w_planes=6).to(dtype=torch.float32)
    j = _job(w)
    g = j["g"]
    ref, rskip, rnorm = _allocating(j)
    grid = torch.zeros(2 * g * g, device="cuda")
    skip = torch.full((1,), 777, dtype=torch.int64, device="cuda")
    norm = torch.full((1,), 0.5, dtype=torch.float64, device="cuda")
    assert _static_call(lib, j, grid, skip, norm) == _lib.OK
    assert _static_status(lib) == _lib.OK
    torch.cuda.synchronize()
    assert int(skip.item()) == rskip
    assert abs(norm.item() - 0.5 - rnorm) <= 1e-12 * abs(rnorm)
    assert rel_rms(grid.cpu().numpy(), ref) <= TOL_F
    # NULL skip count and norm: the grid alone
    grid2 = torch.zeros(2 * g * g, device="cuda")
    assert _static_call(lib, j, grid2, None, None) == _lib.OK
    assert _static_status(lib) == _lib.OK
    torch.cuda.synchronize()
    assert rel_rms(grid2.cpu().numpy(), ref) <= TOL_F
    # no points: skip count reset, norm and grid unchanged
    eref, eskip, enorm = _allocating(j, n=0)
    assert eskip == 0 and enorm == 0.0 and not eref.any()
    grid3 = torch.zeros(2 * g * g, device="cuda")
    skip3 = torch.full((1,), 99, dtype=torch.int64, device="cuda")
    norm3 = torch.full((1,), 2.0, dtype=torch.float64, device="cuda")
    assert _static_call(lib, j, grid3, skip3, norm3, n=0) == _lib.OK
    assert _static_status(lib) == _lib.OK
    torch.cuda.synchronize()
    assert int(skip3.item()) == eskip and norm3.item() == 2.0 + enorm
    assert not grid3.any()
