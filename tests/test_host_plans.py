"""The drop-in's host-side plans, compiled with the host C++ compiler and
checked on the CPU: its band bookkeeping (which rows of the grid are final
after each band of a band-ordered gridding pass, fpga_gridding_b200/csrc/
band_rows.h: every row comes back exactly once and only after every band
that can reach it) and its upload chunks (ingest_plan.h: in order, no gaps
or overlaps, bounded count and sizes, the last chunk about 45 % of the
points)."""
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


def _run_check(tmp_path, name):
    exe = str(tmp_path / name)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", CSRC,
                    os.path.join(HERE, name + ".cpp"), "-o", exe],
                   check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip() == "ok"


@pytest.mark.skipif(shutil.which("g++") is None, reason="no g++")
def test_ingest_chunks_cover_points_in_order(tmp_path):
    _run_check(tmp_path, "ingest_plan_check")
