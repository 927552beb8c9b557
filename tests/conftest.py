import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a B200 (runs the CUDA gridder)")


def golden_names():
    """Gridding fixtures (every fixture but the uniform-weighting ones)."""
    return sorted(os.path.splitext(os.path.basename(p))[0]
                  for p in glob.glob(os.path.join(GOLDEN_DIR, "*.npz"))
                  if not os.path.basename(p).startswith(("weights_", "diag_")))


def load_weights_golden(name):
    """A uniform-weighting fixture: the reference's
    oskar_grid_weights_write then _read on the stored inputs."""
    z = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
    return {k: z[k] for k in z.files}


def load_diag_golden(name):
    """A diagnostics fixture: (inputs dict in the reference convention,
    starting contents of the in/out arrays, the reference's outputs)."""
    z = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
    inputs = dict(num_w_planes=int(z["num_w_planes"]), support=z["support"],
                  oversample=int(z["oversample"]),
                  conv_size_half=int(z["conv_size_half"]),
                  conv_func=z["conv_func"], uu=z["uu"], vv=z["vv"],
                  ww=z["ww"], vis=z["vis"], weight=z["weight"],
                  cell_size_rad=float(z["cell_size_rad"]),
                  w_scale=float(z["w_scale"]), grid_size=int(z["grid_size"]))
    init = {k[5:]: z[k] for k in z.files if k.startswith("init_")}
    init["norm"] = float(init["norm"])
    out = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    out["norm"] = float(out["norm"])
    out["num_skipped"] = int(out["num_skipped"])
    return inputs, init, out


def load_golden(name):
    """A fixture as (inputs dict in the reference convention, outputs)."""
    z = np.load(os.path.join(GOLDEN_DIR, name + ".npz"))
    single = bool(z["single"])
    inputs = dict(num_w_planes=int(z["num_w_planes"]), support=z["support"],
                  oversample=int(z["oversample"]),
                  conv_size_half=int(z["conv_size_half"]),
                  conv_func=z["conv_func"], uu=z["uu"], vv=z["vv"],
                  ww=z["ww"], vis=z["vis"], weight=z["weight"],
                  cell_size_rad=float(z["cell_size_rad"]),
                  w_scale=float(z["w_scale"]), grid_size=int(z["grid_size"]))
    out = dict(grid=z["out_grid"], norm=float(z["out_norm"]),
               skipped=int(z["out_skipped"]), single=single)
    return inputs, out


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.oracle_lib()
    return O
