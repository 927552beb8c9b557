"""The C-ABI library loads, exports exactly what include/*.h declares, and
fails loudly (no CPU fallback) where no sm_100 device is present."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT
import fpga_gridding_b200 as fg
from fpga_gridding_b200 import _lib


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = "\n".join(l for l in text.splitlines()
                         if not l.lstrip().startswith("#"))
        for m in re.finditer(r"OSKAR_B200_EXPORT\s+[\w\s\*]*?\b(\w+)\s*\(",
                             text):
            names.add(m.group(1))
    return names


def test_header_declares_exactly_the_exported_list():
    assert declared_symbols() == set(_lib.EXPORTED_SYMBOLS)


def test_library_loads_and_exports_every_declared_symbol():
    lib = fg.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    info = lib.oskar_b200_build_info().decode()
    assert "sm_100a" in info


def test_library_exports_nothing_else():
    out = os.popen(f"nm -D --defined-only {_lib.LIB_PATH}").read()
    exported = {line.split()[-1] for line in out.splitlines()
                if line.split() and line.split()[-2] == "T"}
    assert exported == set(_lib.EXPORTED_SYMBOLS)


def test_drop_in_signatures_match_reference_header():
    """Same parameter list as oskar_grid_wproj.h:69-86 / 114-131."""
    text = open(os.path.join(ROOT, "include",
                             "oskar_grid_wproj_b200.h")).read()
    for suffix, real in (("d", "double"), ("f", "float")):
        m = re.search(r"void oskar_grid_wproj_%s\((.*?)\);" % suffix, text,
                      re.S)
        params = [" ".join(p.split()) for p in m.group(1).split(",")]
        assert params == [
            "const size_t num_w_planes", "const int* support",
            "const int oversample", "const int conv_size_half",
            f"const {real}* conv_func", "const size_t num_points",
            f"const {real}* uu", f"const {real}* vv", f"const {real}* ww",
            f"const {real}* vis", f"const {real}* weight",
            f"const {real} cell_size_rad", f"const {real} w_scale",
            "const int grid_size", "size_t* num_skipped", "double* norm",
            f"{real}* grid"]


def test_diagnostics_signature_matches_reference_definition():
    """Same parameter list as oskar_grid_wproj_f_diagnostics
    (oskar_grid_wproj.c:245-267), which no reference header declares."""
    text = open(os.path.join(ROOT, "include",
                             "oskar_grid_wproj_b200.h")).read()
    m = re.search(r"void oskar_grid_wproj_f_diagnostics\((.*?)\);", text,
                  re.S)
    params = [" ".join(p.split()) for p in m.group(1).split(",")]
    assert params == [
        "const size_t num_w_planes", "const int* support",
        "const int oversample", "const int conv_size_half",
        "const float* conv_func", "const size_t num_points",
        "const float* uu", "const float* vv", "const float* ww",
        "const float* vis", "const float* weight",
        "const float cell_size_rad", "const float w_scale",
        "const int grid_size", "size_t* num_skipped", "double* norm",
        "float* grid", "long long int* num_vis_per_wsupport",
        "long long int* num_vis_per_wplane", "long long int* num_vis_per_grid",
        "float* avg_wsupport_per_grid", "float* avg_wplane_per_grid"]


def _has_sm100():
    try:
        import torch
        return torch.cuda.is_available() and \
            torch.cuda.get_device_capability(0)[0] == 10
    except Exception:
        return False


@pytest.mark.skipif(_has_sm100(), reason="a B200 is present")
def test_drop_in_fails_loudly_without_a_device():
    """No GPU: the drop-in reports NO_DEVICE and leaves grid/norm alone;
    nothing is computed on the CPU."""
    g = 8
    grid = np.full(2 * g * g, 7.0)
    support = np.array([1], np.int32)
    cube = np.ones(1 * 7 * 7 * 2)
    pts = np.zeros(3)
    with pytest.raises(fg.GridderError) as e:
        fg.oskar_grid_wproj_d(1, support, 4, 7, cube, 3, pts, pts, pts,
                              np.zeros(6), np.ones(3), 1.0 / g, 1.0, g, 5.0,
                              grid)
    assert e.value.status == _lib.ERR_NO_DEVICE
    assert (grid == 7.0).all()


@pytest.mark.skipif(_has_sm100(), reason="a B200 is present")
def test_diagnostics_fails_loudly_without_a_device():
    """No GPU: the diagnostics drop-in reports NO_DEVICE and leaves every
    output alone."""
    g = 8
    grid = np.full(2 * g * g, 7.0, np.float32)
    counts = [np.full(2, 3, np.int64), np.full(2, 3, np.int64),
              np.full(g * g, 3, np.int64)]
    avg = np.full(g * g, 2.0, np.float32)
    pts = np.zeros(3, np.float32)
    with pytest.raises(fg.GridderError) as e:
        fg.oskar_grid_wproj_f_diagnostics(
            1, np.array([1], np.int32), 4, 7, np.ones(98, np.float32), 3,
            pts, pts, pts, np.zeros(6, np.float32), None, 1.0 / g, 1.0, g,
            5.0, grid, *counts, avg, None)
    assert e.value.status == _lib.ERR_NO_DEVICE
    assert (grid == 7.0).all() and (avg == 2.0).all()
    assert all((c == 3).all() for c in counts)


def test_diagnostics_wrapper_refuses_arrays_too_small():
    """The Python wrapper checks the count arrays against the entries the
    reference's indexing needs (largest unclamped plane index in float
    arithmetic) before the library could write past them."""
    g = 8
    ww = np.array([0.0, 24.5, 3.9], np.float32)   # planes 0, 5 (4.95), 2
    pts = np.zeros(3, np.float32)
    args = (1, np.array([1], np.int32), 4, 7, np.ones(98, np.float32), 3,
            pts, pts, ww, np.zeros(6, np.float32), None, 1.0 / g, 1.0, g,
            0.0, np.zeros(2 * g * g, np.float32))
    with pytest.raises(ValueError, match="num_vis_per_wplane"):
        fg.oskar_grid_wproj_f_diagnostics(
            *args, np.zeros(2, np.int64), np.zeros(5, np.int64),
            np.zeros(g * g, np.int64), np.zeros(g * g, np.float32), None)
    with pytest.raises(ValueError, match="num_vis_per_grid"):
        fg.oskar_grid_wproj_f_diagnostics(
            *args, np.zeros(2, np.int64), np.zeros(6, np.int64),
            np.zeros(g * g - 1, np.int64), np.zeros(g * g, np.float32), None)


def test_invalid_arguments_rejected_before_any_device_work():
    lib = fg.load()
    skipped = C.c_size_t(99)
    norm = C.c_double(1.0)
    # null grid
    lib.oskar_grid_wproj_d(1, np.array([1], np.int32).ctypes.data, 4, 6,
                           np.ones(72).ctypes.data, 0, None, None, None,
                           None, None, 0.1, 1.0, 8, C.byref(skipped),
                           C.byref(norm), None)
    assert lib.oskar_grid_wproj_b200_last_error() == _lib.ERR_INVALID_ARGUMENT
    # kernel cube too small for the support: the reference would read past
    # the end of conv_func (oskar_grid_wproj.c:110-116)
    g = np.zeros(128)
    lib.oskar_grid_wproj_d(1, np.array([3], np.int32).ctypes.data, 4, 6,
                           np.ones(72).ctypes.data, 0, None, None, None,
                           None, None, 0.1, 1.0, 8, C.byref(skipped),
                           C.byref(norm), g.ctypes.data)
    assert lib.oskar_grid_wproj_b200_last_error() == _lib.ERR_INVALID_ARGUMENT
    assert norm.value == 1.0


def test_fail_allocation_arms_and_rejects_bad_argument():
    """The allocation-failure testing aid takes a count or -1 (disarm); it
    touches no device."""
    lib = _lib.load()
    assert lib.oskar_b200_testing_fail_allocation(-2) == \
        _lib.ERR_INVALID_ARGUMENT
    assert lib.oskar_b200_testing_fail_allocation(3) == _lib.OK
    assert lib.oskar_b200_testing_fail_allocation(-1) == _lib.OK
