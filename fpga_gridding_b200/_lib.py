"""ctypes binding of libgridder_b200.so (the C ABI in
include/oskar_grid_wproj_b200.h).  Loading fails loudly when the library
has not been built: there is no CPU fallback."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgridder_b200.so")

# Every symbol include/oskar_grid_wproj_b200.h declares.
EXPORTED_SYMBOLS = (
    "oskar_grid_wproj_d",
    "oskar_grid_wproj_f",
    "oskar_grid_wproj_f_diagnostics",
    "oskar_grid_weights_write_d",
    "oskar_grid_weights_read_d",
    "oskar_grid_weights_write_f",
    "oskar_grid_weights_read_f",
    "oskar_grid_wproj_b200_last_error",
    "oskar_grid_wproj_b200_error_string",
    "oskar_grid_wproj_b200_release_thread_cache",
    "oskar_b200_options_init",
    "oskar_b200_workspace_create",
    "oskar_b200_workspace_free",
    "oskar_b200_workspace_bytes",
    "oskar_b200_cube_create",
    "oskar_b200_cube_create_planar",
    "oskar_b200_cube_free",
    "oskar_b200_cube_bytes",
    "oskar_b200_grid",
    "oskar_b200_grid_batch",
    "oskar_b200_degrid",
    "oskar_b200_degrid_host",
    "oskar_b200_place",
    "oskar_b200_weights_write",
    "oskar_b200_weights_read",
    "oskar_b200_blocks_create",
    "oskar_b200_blocks_push",
    "oskar_b200_blocks_finish",
    "oskar_b200_blocks_free",
    "oskar_b200_last_stats",
    "oskar_b200_set_stage_timing",
    "oskar_b200_autotune",
    "oskar_b200_tune_table",
    "oskar_b200_tune_launch",
    "oskar_b200_measure_atomic_rate",
    "oskar_b200_grid_f_static",
    "oskar_b200_grid_f_static_status",
    "oskar_b200_server_create",
    "oskar_b200_server_submit",
    "oskar_b200_server_poll",
    "oskar_b200_server_release",
    "oskar_b200_server_clock",
    "oskar_b200_server_memory",
    "oskar_b200_server_free",
    "oskar_b200_selftest_bounded_wait",
    "oskar_b200_testing_fail_allocation",
    "oskar_b200_testing_set_static_status",
    "oskar_b200_build_info",
)

# Status codes (oskar_B200Status).
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_NO_DEVICE = 2
ERR_OUT_OF_MEMORY = 3
ERR_CUDA = 4
ERR_UNSUPPORTED = 5
ERR_DEVICE_CHECK = 6
ERR_TIMEOUT = 7
ERR_OVER_BUDGET = 8

COORDS_F64 = 0
COORDS_REFERENCE_F32 = 1
KERNEL_NATIVE = 0
KERNEL_F16 = 1
KERNEL_BF16 = 2
ACCUM_PLAIN = 0
ACCUM_COMPENSATED = 1


class Options(C.Structure):
    _fields_ = [("coord_mode", C.c_int), ("kernel_type", C.c_int),
                ("accum_mode", C.c_int), ("apply_weight", C.c_int),
                ("classes_per_thread", C.c_int), ("staging", C.c_int),
                ("compensate_radius", C.c_int), ("tile_shift", C.c_int),
                ("frequency_hz", C.c_double), ("reserved", C.c_int * 6)]


class Stats(C.Structure):
    _fields_ = [("num_points", C.c_ulonglong), ("num_gridded", C.c_ulonglong),
                ("grid_updates", C.c_ulonglong), ("num_tasks", C.c_ulonglong),
                ("atomic_flushes", C.c_ulonglong), ("status", C.c_int),
                ("kernel_launches", C.c_int), ("prep_ms", C.c_float),
                ("sort_ms", C.c_float), ("tasks_ms", C.c_float),
                ("grid_ms", C.c_float)]


_P = C.c_void_p
_SZ = C.c_size_t
_lib = None


class Request(C.Structure):
    """oskar_B200Request: one job submitted to a server."""
    _fields_ = [("tag", C.c_ulonglong), ("cube", _P), ("num_points", _SZ),
                ("uu", _P), ("vv", _P), ("ww", _P), ("vis", _P),
                ("weight", _P), ("cell_size_rad", C.c_double),
                ("w_scale", C.c_double), ("grid_size", C.c_int),
                ("frequency_hz", C.c_double)]


class Completion(C.Structure):
    """oskar_B200Completion."""
    _fields_ = [("tag", C.c_ulonglong), ("status", C.c_int),
                ("num_skipped", C.c_ulonglong), ("norm", C.c_double),
                ("grid", _P), ("submit_s", C.c_double),
                ("start_s", C.c_double), ("end_s", C.c_double),
                ("batch_size", C.c_int)]


class Job(C.Structure):
    """oskar_B200Job: one job of oskar_b200_grid_batch."""
    _fields_ = [("cube", _P), ("num_points", _SZ), ("uu", _P), ("vv", _P),
                ("ww", _P), ("vis", _P), ("weight", _P),
                ("cell_size_rad", C.c_double), ("w_scale", C.c_double),
                ("grid_size", C.c_int), ("grid", _P), ("d_num_skipped", _P),
                ("d_norm", _P), ("frequency_hz", C.c_double)]


def load():
    """The gridder library (raises RuntimeError if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with "
            "`make -C fpga_gridding_b200/csrc` (or __graft_entry__.build())")
    lib = C.CDLL(LIB_PATH)
    grid_common = [_SZ, _P, C.c_int, C.c_int, _P, _SZ, _P, _P, _P, _P, _P]
    lib.oskar_grid_wproj_d.argtypes = grid_common + [
        C.c_double, C.c_double, C.c_int, _P, _P, _P]
    lib.oskar_grid_wproj_f.argtypes = grid_common + [
        C.c_float, C.c_float, C.c_int, _P, _P, _P]
    lib.oskar_grid_wproj_d.restype = lib.oskar_grid_wproj_f.restype = None
    lib.oskar_grid_wproj_f_diagnostics.argtypes = grid_common + [
        C.c_float, C.c_float, C.c_int, _P, _P, _P, _P, _P, _P, _P, _P]
    lib.oskar_grid_wproj_f_diagnostics.restype = None
    for t, real in (("d", C.c_double), ("f", C.c_float)):
        fw = getattr(lib, "oskar_grid_weights_write_" + t)
        fw.argtypes = [_SZ, _P, _P, _P, real, C.c_int, _P, _P]
        fw.restype = None
        fr = getattr(lib, "oskar_grid_weights_read_" + t)
        fr.argtypes = [_SZ, _P, _P, _P, _P, real, C.c_int, _P, _P]
        fr.restype = None
    lib.oskar_b200_weights_write.argtypes = [
        _P, C.c_int, C.c_int, _SZ, _P, _P, _P, C.c_double, C.c_int, _P, _P,
        C.c_double, _P]
    lib.oskar_b200_weights_read.argtypes = [
        _P, C.c_int, _SZ, _P, _P, _P, _P, C.c_double, C.c_int, _P, _P,
        C.c_double, _P]
    lib.oskar_b200_blocks_create.argtypes = [
        _P, _P, C.POINTER(Options), C.c_double, C.c_double, C.c_int, _P, _P,
        C.POINTER(_P)]
    lib.oskar_b200_blocks_push.argtypes = [_P, _SZ, _P, _P, _P, _P, _P,
                                           C.c_double]
    lib.oskar_b200_blocks_finish.argtypes = [_P, C.POINTER(C.c_ulonglong)]
    lib.oskar_b200_blocks_free.argtypes = [_P]
    lib.oskar_grid_wproj_b200_last_error.restype = C.c_int
    lib.oskar_grid_wproj_b200_error_string.argtypes = [C.c_int]
    lib.oskar_grid_wproj_b200_error_string.restype = C.c_char_p
    lib.oskar_grid_wproj_b200_release_thread_cache.restype = None
    lib.oskar_b200_options_init.argtypes = [C.POINTER(Options)]
    lib.oskar_b200_options_init.restype = None
    lib.oskar_b200_workspace_create.argtypes = [C.c_int, C.POINTER(_P)]
    lib.oskar_b200_workspace_free.argtypes = [_P]
    lib.oskar_b200_workspace_bytes.argtypes = [_P]
    lib.oskar_b200_workspace_bytes.restype = _SZ
    lib.oskar_b200_cube_create.argtypes = [
        _P, _SZ, _P, C.c_int, C.c_int, _P, C.c_int, C.c_int, C.c_int,
        C.c_int, _P, C.POINTER(_P)]
    lib.oskar_b200_cube_create_planar.argtypes = [
        _P, _SZ, _P, C.c_int, C.c_int, _P, _P, C.c_int, C.c_int, C.c_int,
        C.c_int, _P, C.POINTER(_P)]
    lib.oskar_b200_degrid.argtypes = [
        _P, _P, C.POINTER(Options), _SZ, _P, _P, _P, _P, C.c_double,
        C.c_double, C.c_int, _P, _P, _P, _P]
    lib.oskar_b200_degrid_host.argtypes = [
        _P, _P, C.POINTER(Options), _SZ, _P, _P, _P, _P, C.c_double,
        C.c_double, C.c_int, _P, _P, C.POINTER(_SZ)]
    lib.oskar_b200_cube_free.argtypes = [_P]
    lib.oskar_b200_cube_bytes.argtypes = [_P]
    lib.oskar_b200_cube_bytes.restype = _SZ
    lib.oskar_b200_grid.argtypes = [
        _P, _P, C.POINTER(Options), _SZ, _P, _P, _P, _P, _P, C.c_double,
        C.c_double, C.c_int, _P, _P, _P, _P]
    lib.oskar_b200_place.argtypes = [
        _P, C.c_int, C.c_int, _SZ, _P, C.c_int, _SZ, _P, _P, _P, C.c_double,
        C.c_double, C.c_int] + [_P] * 7 + [_P]
    lib.oskar_b200_last_stats.argtypes = [_P, C.POINTER(Stats)]
    lib.oskar_b200_build_info.restype = C.c_char_p
    lib.oskar_b200_set_stage_timing.argtypes = [_P, C.c_int]
    lib.oskar_b200_autotune.argtypes = [
        _P, _P, C.POINTER(Options), _SZ, _P, _P, _P, _P, C.c_double,
        C.c_double, C.c_int, _P, _P]
    lib.oskar_b200_tune_table.argtypes = [_P, _P, _P]
    lib.oskar_b200_tune_launch.argtypes = [_P, _P, _P]
    lib.oskar_b200_tune_launch.restype = C.c_int
    lib.oskar_b200_measure_atomic_rate.argtypes = [
        _P, _P, C.c_int, C.c_int, C.POINTER(C.c_double)]
    lib.oskar_b200_grid_batch.argtypes = [_P, C.POINTER(Options), C.c_int,
                                          C.POINTER(Job), _P]
    lib.oskar_b200_grid_f_static.argtypes = [
        _SZ, _P, C.c_int, C.c_int, _P, _SZ, _P, _P, _P, _P, C.c_float,
        C.c_float, C.c_int, _P, _P, _P, _P]
    lib.oskar_b200_grid_f_static.restype = C.c_int
    lib.oskar_b200_grid_f_static_status.argtypes = [_P, C.POINTER(C.c_int)]
    lib.oskar_b200_grid_f_static_status.restype = C.c_int
    lib.oskar_b200_testing_set_static_status.argtypes = [C.c_ulonglong, _P]
    lib.oskar_b200_testing_set_static_status.restype = C.c_int
    lib.oskar_b200_testing_fail_allocation.argtypes = [C.c_longlong]
    lib.oskar_b200_testing_fail_allocation.restype = C.c_int
    lib.oskar_b200_selftest_bounded_wait.argtypes = [_P, C.c_uint,
                                                     C.POINTER(C.c_int)]
    lib.oskar_b200_selftest_bounded_wait.restype = C.c_int
    lib.oskar_b200_server_create.argtypes = [C.c_int, _SZ, C.c_int, C.c_int,
                                             C.POINTER(Options),
                                             C.POINTER(_P)]
    lib.oskar_b200_server_submit.argtypes = [_P, C.POINTER(Request)]
    lib.oskar_b200_server_poll.argtypes = [_P, C.POINTER(Completion), C.c_int,
                                           C.POINTER(C.c_int), C.c_double]
    lib.oskar_b200_server_release.argtypes = [_P, C.c_ulonglong]
    lib.oskar_b200_server_clock.argtypes = [_P]
    lib.oskar_b200_server_clock.restype = C.c_double
    lib.oskar_b200_server_memory.argtypes = [_P, C.POINTER(_SZ),
                                             C.POINTER(_SZ)]
    lib.oskar_b200_server_free.argtypes = [_P]
    for name in ("oskar_b200_server_create", "oskar_b200_server_submit",
                 "oskar_b200_server_poll", "oskar_b200_server_release",
                 "oskar_b200_server_memory", "oskar_b200_server_free"):
        getattr(lib, name).restype = C.c_int
    for name in ("oskar_b200_workspace_create", "oskar_b200_workspace_free",
                 "oskar_b200_cube_create", "oskar_b200_cube_free",
                 "oskar_b200_grid", "oskar_b200_grid_batch",
                 "oskar_b200_place", "oskar_b200_last_stats",
                 "oskar_b200_set_stage_timing",
    "oskar_b200_autotune",
    "oskar_b200_tune_table",
                 "oskar_b200_measure_atomic_rate"):
        getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib


class GridderError(RuntimeError):
    def __init__(self, status: int, where: str = ""):
        msg = load().oskar_grid_wproj_b200_error_string(status).decode()
        super().__init__(f"{where}: status {status} ({msg})" if where else
                         f"status {status} ({msg})")
        self.status = status


def check(status: int, where: str = "") -> None:
    if status != OK:
        raise GridderError(status, where)
