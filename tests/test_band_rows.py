"""The drop-in's band bookkeeping (which rows of the grid are final after
each band of a band-ordered gridding pass, fpga_gridding_b200/csrc/
band_rows.h), compiled with the host C++ compiler and checked on many band
layouts: every row comes back exactly once and only after every band that
can reach it.  Runs on the CPU."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "fpga_gridding_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_final_rows_every_row_once_after_its_bands(tmp_path):
    exe = str(tmp_path / "band_rows_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", CSRC,
                    os.path.join(HERE, "band_rows_check.cpp"), "-o", exe],
                   check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"
