"""Placement parity at the benchmark sizes: every visibility of the full
plain_large job (39,244,800 points, 8192^2 grid, 256 w-planes) and of the
lowest and highest batch128 channels is placed on the GPU
(oskar_b200_place, which runs the same place_one as the gridding prep) and
by the CPU oracle, which restates oskar_grid_wproj.c:70-101 and is pinned
bit-exact to the compiled reference.  Bar: num_skipped and every kept
visibility's (grid_u, grid_v, w-plane, off_u, off_v, conj) bit-exact, for
the FP32 inputs the benchmark grids (FP64 placement of the float values) and
for the same job in FP64."""
import numpy as np
import pytest
import torch

import fpga_gridding_b200 as fg
from fpga_gridding_b200 import _lib, workloads as W

pytestmark = pytest.mark.gpu

FIELDS = ("gu", "gv", "plane", "off_u", "off_v", "conj")


@pytest.fixture(scope="module")
def ws():
    w = fg.Workspace(0)
    yield w
    w.close()


def _host(w, single):
    """The inputs as the oracle sees them: for an FP32 job, the float values
    held in float64, and cell / w_scale rounded to float as the FP32 entry
    points receive them."""
    d = dict(num_w_planes=w.num_w_planes, support=w.support,
             oversample=w.oversample, grid_size=w.grid_size)
    for k in ("uu", "vv", "ww"):
        a = getattr(w, k).cpu().numpy()
        d[k] = a.astype(np.float32).astype(np.float64) if single else a
    cast = (lambda x: float(np.float32(x))) if single else float
    d["cell_size_rad"] = cast(w.cell_size_rad)
    d["w_scale"] = cast(w.w_scale)
    return d


def _check_every_visibility(ws, oracle, w, single):
    dt = torch.float32 if single else torch.float64
    h = _host(w, single)
    got = fg.place_device(ws, w.support, w.oversample,
                          w.uu.to(dtype=dt, device="cuda"),
                          w.vv.to(dtype=dt, device="cuda"),
                          w.ww.to(dtype=dt, device="cuda"),
                          h["cell_size_rad"], h["w_scale"], w.grid_size,
                          coord_mode=_lib.COORDS_F64)
    torch.cuda.synchronize()
    got = {k: v.cpu().numpy() for k, v in got.items()}
    ref = oracle.place(h)
    n = len(h["uu"])
    assert got["skipped"].shape[0] == n
    skip_mismatch = int(np.count_nonzero(
        got["skipped"] != ref["skipped"].astype(np.int32)))
    assert skip_mismatch == 0, f"{skip_mismatch} skip flags differ"
    keep = ref["skipped"] == 0
    for k in FIELDS:
        bad = int(np.count_nonzero(got[k][keep] !=
                                   ref[k][keep].astype(np.int32)))
        assert bad == 0, f"{bad} of {int(keep.sum())} values of {k} differ"
    return n


def test_plain_large_every_placement_bit_exact(ws, oracle):
    w = W.plain_large(seed=1, device="cuda")
    assert w.num_points == 39_244_800
    for single in (True, False):
        assert _check_every_visibility(ws, oracle, w, single) == 39_244_800
    del w
    torch.cuda.empty_cache()


def test_batch128_lowest_and_highest_channel_placements_bit_exact(ws, oracle):
    chans = W.batch_channels(seed=2, device="cuda")
    assert len(chans) == 128
    for c in (chans[0], chans[-1]):
        _check_every_visibility(ws, oracle, c, True)
    del chans
    torch.cuda.empty_cache()
