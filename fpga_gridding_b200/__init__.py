"""B200-native W-projection gridder (drop-in for the reference's
oskar_grid_wproj_d / oskar_grid_wproj_f).

The product is the C-ABI library libgridder_b200.so (hand-written sm_100a
CUDA, declared in include/oskar_grid_wproj_b200.h); this package is its
Python front end.  Importing the package does not load the library;
calling any gridding function does, and fails loudly if it is missing.
"""
from ._lib import EXPORTED_SYMBOLS, GridderError, LIB_PATH, load  # noqa: F401
from .gridder import (Blocks, Cube, Workspace, degrid_device, degrid_host, grid_batch_device, grid_device,  # noqa: F401
                      grid_workload,
                      options, oskar_grid_weights_read_d,
                      oskar_grid_weights_read_f, oskar_grid_weights_write_d,
                      oskar_grid_weights_write_f, oskar_grid_wproj_d,
                      oskar_grid_wproj_f, oskar_grid_wproj_f_diagnostics,
                      place_device, weights_read_device,
                      weights_write_device)
