"""Failure detection on the device without a GPU fault: every device-side
wait of the gridder is bounded, and an expired wait becomes a status the
host reads.  The self-test kernel waits on a barrier phase that nothing
completes; the test checks the timeout status and that the same workspace
then grids correctly (the context stayed usable)."""
import ctypes as C

import numpy as np
import pytest

import fpga_gridding_b200 as fg
from fpga_gridding_b200 import _lib, workloads as W

pytestmark = pytest.mark.gpu


def test_bounded_wait_expires_with_status(oracle):
    ws = fg.Workspace(0)
    try:
        lib = _lib.load()
        st = C.c_int(-1)
        rc = lib.oskar_b200_selftest_bounded_wait(ws.handle, 256,
                                                  C.byref(st))
        assert rc == _lib.OK
        assert st.value == _lib.ERR_TIMEOUT
        # The context is still usable: a drop-in call after the expired
        # wait matches the oracle.
        w = W.plain_small().numpy()
        s1, n1, g1 = oracle.grid_d(w, threads=8)
        s2, n2, g2 = fg.grid_workload(w, single=False)
        assert s2 == s1
        assert oracle.rel_rms(g2, g1) <= 1e-12
    finally:
        ws.close()


def test_bounded_wait_rejects_bad_arguments():
    ws = fg.Workspace(0)
    try:
        lib = _lib.load()
        st = C.c_int(0)
        assert lib.oskar_b200_selftest_bounded_wait(
            ws.handle, 0, C.byref(st)) == _lib.ERR_INVALID_ARGUMENT
        assert lib.oskar_b200_selftest_bounded_wait(
            None, 16, C.byref(st)) == _lib.ERR_INVALID_ARGUMENT
    finally:
        ws.close()


def _dropin_d(w, grid, norm):
    """oskar_grid_wproj_d through ctypes; returns (status, skipped, norm)."""
    lib = _lib.load()
    a = {k: np.ascontiguousarray(w[k], np.float64)
         for k in ("conv_func", "uu", "vv", "ww", "vis", "weight")}
    sup = np.ascontiguousarray(w["support"], np.int32)
    sk, nrm = C.c_size_t(12345), C.c_double(norm)
    lib.oskar_grid_wproj_d(w["num_w_planes"], sup.ctypes.data,
                           w["oversample"], w["conv_size_half"],
                           a["conv_func"].ctypes.data, len(a["uu"]),
                           a["uu"].ctypes.data, a["vv"].ctypes.data,
                           a["ww"].ctypes.data, a["vis"].ctypes.data,
                           a["weight"].ctypes.data, w["cell_size_rad"],
                           w["w_scale"], w["grid_size"], C.byref(sk),
                           C.byref(nrm), grid.ctypes.data)
    return lib.oskar_grid_wproj_b200_last_error(), sk.value, nrm.value


@pytest.mark.parametrize("after", [0, 2, 5, 20])
def test_dropin_allocation_failure_leaves_grid_and_norm(after):
    """A device allocation that fails (injected on the host: the after-th
    next allocation of the library reports out-of-memory) makes the drop-in
    report OSKAR_B200_ERR_OUT_OF_MEMORY with the caller's grid and norm
    untouched; the next call, with nothing injected, grids normally."""
    lib = _lib.load()
    w = W.plain_small().numpy()
    g = w["grid_size"]
    base = np.random.default_rng(8).normal(size=2 * g * g)
    # a fresh per-thread workspace: the next call allocates its buffers
    lib.oskar_grid_wproj_b200_release_thread_cache()
    assert lib.oskar_b200_testing_fail_allocation(after) == _lib.OK
    try:
        grid = base.copy()
        st, _, nrm = _dropin_d(w, grid, 2.5)
    finally:
        lib.oskar_b200_testing_fail_allocation(-1)
    assert st == _lib.ERR_OUT_OF_MEMORY
    assert nrm == 2.5
    assert np.array_equal(grid, base)
    grid2 = base.copy()
    st2, sk2, n2 = _dropin_d(w, grid2, 2.5)
    grid3 = base.copy()
    st3, sk3, n3 = _dropin_d(w, grid3, 2.5)
    assert st2 == _lib.OK and st3 == _lib.OK
    assert sk2 == sk3 and abs(n2 - n3) <= 1e-12 * abs(n3)
    assert np.abs(grid2 - grid3).max() <= 1e-9 * np.abs(grid3).max()
    assert not np.array_equal(grid2, base)
