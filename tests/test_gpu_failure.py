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
