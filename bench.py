#!/usr/bin/env python
"""Benchmark of the B200 W-projection gridder on the large single-job
workload (plain_large: 39,244,800 visibilities onto an 8192^2 complex64
grid, 256 w-planes with support 4..36, oversample 4, FP32 data, kernels and
grid, FP64 coordinates).

A step grids the whole job once.  `value` is visibilities per second (Gvis/s)
with inputs resident in HBM, timed with CUDA events on the launching stream
over exactly --steps steps after --warmup untimed steps; the inputs (0.8 GB
per step) are larger than L2, so no flush is needed between steps.  `e2e` is
the same metric through the drop-in C entry point oskar_grid_wproj_f with
pinned host buffers (host<->device copies inside the timed region).

Multi-GPU (torchrun, one process per GPU): every rank grids its own
independent job (different seed) with no collective on the data path; the
elapsed time is the max over ranks (weak scaling).

--impl reference times the reference's own CPU gridder (oskar_grid_wproj.c
compiled unmodified into oracle/_ref, driven in its fixed 10000-point calls
over a bounded random sample of the same workload) on all host cores.
"""
from __future__ import annotations

import argparse
import datetime
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402

METRIC = ("Gvis/s & grid updates/s at ≤1e-5 rel err vs FP64; "
          "serving p50/p99 latency")
UNIT = "Gvis/s"
WORKLOAD_DESC = ("plain_large: 512 stations log-radial to 30 km (130,816 "
                 "baselines) x 300 samples = 39,244,800 visibilities, 150 MHz, "
                 "dec -30 deg; grid 8192^2 complex64; 256 w-planes, support "
                 "4->36, oversample 4, conv_size_half 149; FP32 data/kernels/"
                 "grid, FP64 coordinates")
DATA_DESC = ("synthetic: seeded Earth-rotation uvw, 10 point sources + "
             "complex Gaussian noise, analytic Gaussian x chirp W-kernels")
FALLBACK_HBM_GBS = 6650.0


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def dist_setup(gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    from fpga_gridding_b200 import replicas
    return replicas.max_over_ranks(x, world, device="cuda")


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profiled_value(key, profile="romein_grid_kernel_plain_large.md"):
    """A per-launch figure from a committed ncu summary (by default the
    gridding kernel's, profiles/romein_grid_kernel_plain_large.md), or
    None."""
    p = os.path.join(ROOT, "profiles", profile)
    try:
        text = open(p).read()
    except OSError:
        return None
    m = re.search(key + r":\s*([0-9.eE+]+)", text)
    return float(m.group(1)) if m else None


def profiled_traffic():
    """DRAM bytes (read + write) of one full-size gridding launch."""
    return profiled_value("dram_bytes_per_launch_full_job")


def issue_peak_per_s(device=0):
    """Warp instructions the device can issue per second: 4 schedulers per
    SM, one instruction each per cycle, at the maximum SM clock."""
    props = torch.cuda.get_device_properties(device)
    mhz = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            mhz = float(json.load(f)["sm_max_mhz"])
    except Exception:
        out = subprocess.run(["nvidia-smi", "--query-gpu=clocks.max.sm",
                              "--format=csv,noheader,nounits", "-i",
                              str(device)], capture_output=True, text=True)
        try:
            mhz = float(out.stdout.strip().splitlines()[0])
        except (ValueError, IndexError):
            return None
    return props.multi_processor_count * 4 * mhz * 1e6


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200", "-i",
                 str(self.dev)], stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # nvidia-smi's start-up (NVML initialisation) must not overlap the
        # timed region: wait for its first sample.
        t0 = time.time()
        while time.time() - t0 < 10.0 and os.path.getsize(self.path) == 0:
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9])
                          if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def host_threads():
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    return max(1, n)


def mem_available_bytes():
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 16 << 30


def ensure_oracle():
    from oracle import oracle as O
    if not os.path.exists(O.ORACLE_SO):
        O.build()
    return O


def cpu_sample_time(O, wl_host, single, use_reference, target_s, seed,
                    threads=None):
    """Time the reference (or the restatement) on a random sample of the
    workload sized for about target_s seconds on `threads` host threads.
    Returns (seconds, sample_points, grid_updates, threads, kind)."""
    n_all = len(wl_host["uu"])
    g = wl_host["grid_size"]
    grid_bytes = 2 * g * g * (4 if single else 8)
    t = threads or host_threads()
    t = max(1, min(t, int(0.5 * mem_available_bytes() // grid_bytes), 256))
    rng = np.random.default_rng(seed)

    def sample(m):
        idx = np.sort(rng.choice(n_all, size=min(m, n_all), replace=False))
        s = dict(wl_host)
        for k in ("uu", "vv", "ww", "weight"):
            s[k] = wl_host[k][idx]
        s["vis"] = wl_host["vis"].reshape(-1, 2)[idx].reshape(-1)
        return s
    # calibrate the per-thread rate on a small sample
    cal = sample(20000 * t)
    secs, _, _, _ = O.time_parallel(cal, single, t, use_reference)
    rate = len(cal["uu"]) / max(secs, 1e-6)
    m = int(max(10000 * t, rate * target_s))
    s = sample(m)
    secs, _, _, _ = O.time_parallel(s, single, t, use_reference)
    taps = O.count_taps(s)
    kind = "reference" if use_reference else "port"
    return secs, len(s["uu"]), taps, t, kind


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------

def make_workload(rank, stations=512):
    """The benchmark job; fewer stations give the smaller profiling case
    (same grid, planes and kernels)."""
    from fpga_gridding_b200 import workloads as W
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    wl = W.plain_large(seed=1 + rank, device=dev, num_stations=stations)
    return wl.to(dtype=torch.float32)


def host_dict(wl32):
    d = wl32.numpy()
    d["cell_size_rad"] = float(np.float32(wl32.cell_size_rad))
    d["w_scale"] = float(np.float32(wl32.w_scale))
    return d


def plain_config(stations, n, g, planes, oversample, world):
    """The `config` of a plain_large line; both arms emit the same keys."""
    workload = WORKLOAD_DESC if stations == 512 else (
        f"profiling case: plain_large with {stations} stations "
        f"({n} visibilities), otherwise identical")
    return {"workload": workload, "num_points": n, "grid_size": g,
            "num_w_planes": planes, "oversample": oversample,
            "parallelism": f"replicas x{world}" if world > 1 else "single",
            "l2": "inputs (0.8 GB/step) larger than L2; no flush"}


def run_b200(args, world, rank, local):
    import ctypes as C
    import fpga_gridding_b200 as fg
    from fpga_gridding_b200 import _lib

    lib = fg.load()
    wl = make_workload(rank, args.stations)
    n = wl.num_points
    g = wl.grid_size
    cell = float(np.float32(wl.cell_size_rad))
    wsc = float(np.float32(wl.w_scale))
    ws = fg.Workspace(local)
    lib.oskar_b200_set_stage_timing(ws.handle, 1)
    cube = fg.Cube(ws, wl.support, wl.oversample, wl.conv_size_half,
                   wl.conv_func, data_is_double=False)
    grid = torch.zeros(2 * g * g, dtype=torch.float32, device="cuda")
    skip = torch.zeros(1, dtype=torch.int64, device="cuda")
    norm = torch.zeros(1, dtype=torch.float64, device="cuda")
    # A real (non-default) stream: the library launches on it and the
    # timing events are recorded on it.
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    opts = fg.options(classes_per_thread=args.cpt)
    tuned = None
    if args.autotune:
        # classes per thread measured per support on a seeded 2 M sample
        rng = np.random.default_rng(5)
        idx = torch.as_tensor(np.sort(rng.choice(n, size=min(n, 2_000_000),
                                                 replace=False)),
                              device="cuda")
        smp = wl.subset(idx)
        tuned = ws.autotune(cube, smp.uu, smp.vv, smp.ww, smp.vis, cell, wsc,
                            g, grid).tolist()
        tuned_launch = dict(zip(("tile_shift", "staging",
                                 "compensate_radius"), ws.tune_launch()))
        grid.zero_()

    def step():
        fg.grid_device(ws, cube, wl.uu, wl.vv, wl.ww, wl.vis, wl.weight,
                       cell, wsc, g, grid, skip, norm, opts=opts,
                       stream=stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    grid_ms, launches, stats = [], 0, None
    ev0.record(stream)
    for _ in range(args.steps):
        step()
        stream.synchronize()  # stage events of this step are now readable
        stats = ws.stats()
        grid_ms.append(stats.grid_ms)
        launches += stats.kernel_launches
        if stats.status != 0:
            raise RuntimeError(f"device check status {stats.status}")
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    elapsed_ms = ev0.elapsed_time(ev1)
    # One more (untimed) step with the grid atomics counted: counting costs
    # an instruction per tap, so the timed steps run without it.
    lib.oskar_b200_set_stage_timing(ws.handle, 3)
    step()
    stream.synchronize()
    issued_atomics = ws.stats().atomic_flushes
    lib.oskar_b200_set_stage_timing(ws.handle, 1)
    barrier(world)
    elapsed_ms = max_over_ranks(elapsed_ms, world)
    ms_per_step = elapsed_ms / args.steps
    total_vis = n * args.steps * world
    value = total_vis / (elapsed_ms * 1e-3) / 1e9
    updates = stats.grid_updates
    updates_per_s = updates * args.steps * world / (elapsed_ms * 1e-3)

    # Roofline of the dominant kernel (the Romein gridding kernel).
    kernel_ms = statistics.mean(grid_ms)
    cube_slab_bytes = cube.bytes
    alg_bytes = n * (16 + 8) + 2 * g * g * 8 + cube_slab_bytes
    achieved = alg_bytes / (kernel_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profiled_traffic()
    # The kernel's ceiling is not HBM: ncu shows instruction issue and the
    # latency of its kernel-value loads limiting it with DRAM nearly idle
    # (profiles/romein_grid_kernel_plain_large.md).  achieved/peak/frac
    # still place its algorithmic bytes against the measured HBM copy rate;
    # the L2-atomic roofline of its grid updates is in "l2_atomic".
    roofline = {"kernel": "romein_grid_kernel<float,float2,L1>",
                "bound": "issue",
                "bound_evidence": "ncu small case: issue slots and "
                                  "kernel-value load latency limit it; "
                                  "DRAM throughput about 1 %",
                "achieved": round(achieved, 2), "peak": peak,
                "peak_source": peak_kind, "unit": "GB/s",
                "frac": round(achieved / peak, 4),
                "traffic": traffic,
                "traffic_source": "ncu dram__bytes_read.sum + "
                                  "dram__bytes_write.sum of one full-size "
                                  "launch, copied from profiles/"
                                  "romein_grid_kernel_plain_large.md (not "
                                  "measured in this run)",
                "algorithmic_bytes_per_launch": alg_bytes,
                "kernel_ms": round(kernel_ms, 3)}
    # The ceiling that binds: instruction issue.  Warp instructions of one
    # full-size launch (ncu smsp__inst_executed.sum, copied from the
    # profile) over this run's kernel time, against the issue rate.
    winst = profiled_value("warp_instructions_per_launch_full_job")
    ipeak = issue_peak_per_s(local)
    if winst and ipeak:
        roofline["issue"] = {
            "achieved_warp_inst_per_s": winst / (kernel_ms * 1e-3),
            "peak_warp_inst_per_s": ipeak,
            "frac": round(winst / (kernel_ms * 1e-3) / ipeak, 4),
            "warp_instructions_per_launch": winst,
            "source": "ncu smsp__inst_executed.sum of one full-size launch, "
                      "copied from profiles/romein_grid_kernel_plain_large.md"
                      "; peak = SMs x 4 schedulers x max SM clock"}
    # L2-atomic roofline: measured complex-FP32 red.v2 rate on an
    # L2-resident 2048^2 grid.
    rate = C.c_double(0.0)
    probe = torch.zeros(2 * 2048 * 2048, dtype=torch.float32, device="cuda")
    _lib.check(lib.oskar_b200_measure_atomic_rate(
        ws.handle, C.c_void_p(probe.data_ptr()), 2048, 2000, C.byref(rate)))
    del probe
    kernel_updates_per_s = updates / (kernel_ms * 1e-3)
    l2_atomic = {"peak_red_v2_per_s": rate.value,
                 "grid_updates_per_s_in_kernel": kernel_updates_per_s,
                 "frac": round(kernel_updates_per_s / rate.value, 4),
                 "issued_atomics_per_launch": issued_atomics,
                 "issued_atomic_frac": round(
                     issued_atomics / (kernel_ms * 1e-3) / rate.value, 4)}
    stage_ms = {"prep": round(stats.prep_ms, 3), "sort": round(stats.sort_ms, 3),
                "tasks": round(stats.tasks_ms, 3),
                "grid": round(stats.grid_ms, 3)}

    # End to end through the drop-in C entry point with pinned host buffers.
    e2e = None if args.no_e2e else run_e2e(args, wl, world)

    out = {"metric": METRIC, "value": round(value, 4), "unit": UNIT,
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(ms_per_step, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": DATA_DESC,
           "config": plain_config(args.stations, n, g, wl.num_w_planes,
                                  wl.oversample, world),
           "grid_updates_per_s": updates_per_s,
           "grid_updates_per_step": updates,
           "roofline": roofline, "l2_atomic": l2_atomic, "stage_ms": stage_ms,
           "e2e": e2e, "gpu_launches": launches, "clocks": clk}
    if tuned is not None:
        sup = [int(x) for x in np.unique(wl.support)]
        out["autotuned_classes_per_thread"] = {s: tuned[s] for s in sup}
        out["autotuned_launch"] = tuned_launch
    if rank == 0 and world == 1 and not args.no_cpu_baseline and \
            args.stations == 512:
        out["cpu_baseline"] = run_cpu_baseline(args, wl)
        out["rel_err_vs_fp64"] = audit_error(wl)
    return out


def run_e2e(args, wl, world):
    """Drop-in oskar_grid_wproj_f on pinned host buffers, K steps."""
    import fpga_gridding_b200 as fg
    pin = lambda t: t.cpu().pin_memory()
    h = {k: pin(getattr(wl, k)) for k in ("uu", "vv", "ww", "vis", "weight",
                                          "conv_func")}
    g = wl.grid_size
    hgrid = torch.zeros(2 * g * g, dtype=torch.float32).pin_memory()
    a = {k: v.numpy() for k, v in h.items()}
    gridn = hgrid.numpy()
    cell = float(np.float32(wl.cell_size_rad))
    wsc = float(np.float32(wl.w_scale))

    def call():
        return fg.oskar_grid_wproj_f(
            wl.num_w_planes, wl.support, wl.oversample, wl.conv_size_half,
            a["conv_func"], wl.num_points, a["uu"], a["vv"], a["ww"],
            a["vis"], a["weight"], cell, wsc, g, 0.0, gridn)
    for _ in range(max(1, args.warmup)):
        call()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        call()
    secs = time.perf_counter() - t0
    secs = max_over_ranks(secs, world)
    n = wl.num_points
    h2d = n * 5 * 4 + a["conv_func"].nbytes + gridn.nbytes + wl.num_w_planes * 4
    d2h = gridn.nbytes + 16
    fg.load().oskar_grid_wproj_b200_release_thread_cache()
    return {"value": round(n * args.steps * world / secs / 1e9, 4),
            "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h,
            "ms_per_step": round(1e3 * secs / args.steps, 3),
            "path": "oskar_grid_wproj_f (drop-in C ABI), pinned host buffers"}


def run_cpu_baseline(args, wl):
    O = ensure_oracle()
    use_ref = O.reference_lib() is not None
    hd = host_dict(wl)
    secs, m, taps, t, kind = cpu_sample_time(O, hd, True, use_ref,
                                             args.cpu_seconds, seed=99)
    return {"value": round(m / secs / 1e9, 6), "unit": UNIT, "cores": t,
            "kind": kind, "grid_updates_per_s": taps / secs,
            "sample": (f"{m} visibilities drawn uniformly (seeded) from the "
                       f"39,244,800 of the workload; "
                       + ("reference oskar_grid_wproj_f compiled unmodified, "
                          "driven in its fixed 10000-point calls"
                          if kind == "reference" else
                          "C restatement of oskar_grid_wproj_f")
                       + f"; {t} threads with private 8192^2 grids; "
                       f"{secs:.2f} s")}


def audit_error(wl, m=200000):
    """Relative RMS of the GPU grid vs the FP64 oracle on a seeded sample."""
    import fpga_gridding_b200 as fg
    O = ensure_oracle()
    hd = host_dict(wl)
    rng = np.random.default_rng(7)
    idx = np.sort(rng.choice(len(hd["uu"]), size=m, replace=False))
    s = dict(hd)
    for k in ("uu", "vv", "ww", "weight"):
        s[k] = hd[k][idx]
    s["vis"] = hd["vis"].reshape(-1, 2)[idx].reshape(-1)
    sd = dict(s)
    for k in ("conv_func", "uu", "vv", "ww", "vis", "weight"):
        sd[k] = np.asarray(s[k], np.float64)
    _, n_ref, g_ref = O.grid_d(sd, threads=host_threads())
    _, n_gpu, g_gpu = fg.grid_workload(s, single=True)
    fg.load().oskar_grid_wproj_b200_release_thread_cache()
    return {"grid_rel_rms": O.rel_rms(g_gpu, g_ref),
            "norm_rel": abs(n_gpu - n_ref) / abs(n_ref),
            "sample": f"{m} seeded visibilities of the workload, FP32 drop-in "
                      "vs FP64 oracle on the same inputs"}


BATCH_DESC = ("batch128: 128 channels 50-350 MHz, each into its own 2048^2 "
              "complex64 grid with its own cube (64 w-planes, support 3->24 "
              "scaled by frequency, oversample 4); 256 stations in a 10 km "
              "disk x 60 samples (1,958,400 visibilities per channel before "
              "seeded 0-70% flagging)")


def run_batch128(args, world, rank, local):
    """Batched gridding of 128 uneven channels in one graph-captured
    pipeline (FP32) against the same channels as 128 sequential FP32 jobs;
    the FP16-kernel compensated batch is timed beside it."""
    import ctypes as C
    import fpga_gridding_b200 as fg
    from fpga_gridding_b200 import _lib, workloads as W

    lib = fg.load()
    chans = [c.to(dtype=torch.float32) for c in
             W.batch_channels(seed=2 + rank, device="cuda")]
    n_total = sum(c.num_points for c in chans)
    ws = fg.Workspace(local)
    s = torch.cuda.Stream()
    torch.cuda.synchronize()

    def make_jobs(kernel_type):
        cubes = [fg.Cube(ws, c.support, c.oversample, c.conv_size_half,
                         c.conv_func, data_is_double=False,
                         kernel_type=kernel_type) for c in chans]
        jobs = [dict(cube=cb, uu=c.uu, vv=c.vv, ww=c.ww, vis=c.vis,
                     weight=c.weight,
                     cell_size_rad=float(np.float32(c.cell_size_rad)),
                     w_scale=float(np.float32(c.w_scale)),
                     grid_size=c.grid_size,
                     grid=torch.zeros(2 * c.grid_size ** 2,
                                      dtype=torch.float32, device="cuda"),
                     d_num_skipped=torch.zeros(1, dtype=torch.int64,
                                               device="cuda"),
                     d_norm=torch.zeros(1, dtype=torch.float64, device="cuda"))
                for c, cb in zip(chans, cubes)]
        return cubes, jobs

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        s.synchronize()
        barrier(world)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(args.steps):
            fn()
        e1.record(s)
        e1.synchronize()
        return max_over_ranks(e0.elapsed_time(e1) / args.steps, world)

    # (a) 128 sequential plain FP32 jobs
    cubes32, jobs32 = make_jobs(_lib.KERNEL_NATIVE)
    plain = fg.options()

    def sequential():
        for j in jobs32:
            fg.grid_device(ws, j["cube"], j["uu"], j["vv"], j["ww"], j["vis"],
                           j["weight"], j["cell_size_rad"], j["w_scale"],
                           j["grid_size"], j["grid"], j["d_num_skipped"],
                           j["d_norm"], opts=plain, stream=s)
    seq_ms = timed(sequential)

    # (b) one batch, FP32 plain (the same arithmetic as (a)), captured in a
    # CUDA graph: the headline
    def graph_of(jobs, opts):
        fg.grid_batch_device(ws, jobs, opts=opts, stream=s)  # sizes buffers
        s.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            fg.grid_batch_device(ws, jobs, opts=opts, stream=s)
        return g

    def replay_on_s(g):
        # torch launches a replay on the current stream; keep every use of
        # the workspace's buffers on s.
        def run():
            with torch.cuda.stream(s):
                g.replay()
        return run

    def stage_stats(jobs, opts):
        lib.oskar_b200_set_stage_timing(ws.handle, 1)
        fg.grid_batch_device(ws, jobs, opts=opts, stream=s)
        s.synchronize()
        st = ws.stats()
        lib.oskar_b200_set_stage_timing(ws.handle, 0)
        return st

    g32 = graph_of(jobs32, plain)
    clocks = ClockSampler(local)
    clocks.start()
    batch32_ms = timed(replay_on_s(g32))
    clk = clocks.stop()
    del g32
    st = stage_stats(jobs32, plain)
    err = {}
    if rank == 0 and not args.no_cpu_baseline:
        err = audit_batch(chans, cubes32, ws, plain)
    for cb in cubes32:
        cb.close()
    del jobs32

    # (c) compensation on the heavily hit central cells only: the radius
    # (Chebyshev distance from the grid centre, in cells, tested per task)
    # holding half of all channels' visibilities, where the uv density and
    # hence each cell's running sum are largest.
    radius = central_radius(chans, 0.5)
    comp_c = fg.options(accum_mode=_lib.ACCUM_COMPENSATED,
                        compensate_radius=radius)
    cubes32, jobs32 = make_jobs(_lib.KERNEL_NATIVE)
    gc = graph_of(jobs32, comp_c)
    batch32c_ms = timed(replay_on_s(gc))
    del gc
    err32c = {}
    if rank == 0 and not args.no_cpu_baseline:
        err32c = audit_batch(chans, cubes32, ws, comp_c)
    for cb in cubes32:
        cb.close()
    del jobs32

    # (d) one batch, FP16 kernels + compensated accumulation (whole grid,
    # then central cells), graph-captured
    cubes16, jobs16 = make_jobs(_lib.KERNEL_F16)
    comp = fg.options(accum_mode=_lib.ACCUM_COMPENSATED)
    g16 = graph_of(jobs16, comp)
    batch16_ms = timed(replay_on_s(g16))
    del g16
    g16c = graph_of(jobs16, comp_c)
    batch16c_ms = timed(replay_on_s(g16c))
    del g16c
    err16, err16c = {}, {}
    if rank == 0 and not args.no_cpu_baseline:
        err16 = audit_batch(chans, cubes16, ws, comp)
        err16c = audit_batch(chans, cubes16, ws, comp_c)
    for cb in cubes16:
        cb.close()
    value = n_total * world / (batch32_ms * 1e-3) / 1e9
    return {"metric": METRIC, "value": round(value, 4), "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(batch32_ms, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": DATA_DESC,
            "config": {"workload": BATCH_DESC, "num_points": n_total,
                       "channels": len(chans),
                       "mode": "one graph-captured batch: FP32 kernels and "
                               "grids, plain accumulation",
                       "l2": "inputs (3.9 GB/step) larger than L2; no flush"},
            "sequential_plain_fp32_ms": round(seq_ms, 3),
            "speedup_vs_sequential_plain_fp32": round(seq_ms / batch32_ms, 3),
            "grid_updates_per_s": st.grid_updates * world / (batch32_ms * 1e-3),
            "stage_ms": {"prep": round(st.prep_ms, 3),
                         "sort": round(st.sort_ms, 3),
                         "tasks": round(st.tasks_ms, 3),
                         "grid": round(st.grid_ms, 3)},
            "gpu_launches": st.kernel_launches * args.steps,
            "rel_err_vs_fp64": err,
            "compensate_radius_cells": radius,
            "f32_compensated_central_batch": {
                "ms_per_step": round(batch32c_ms, 3),
                "value": round(n_total * world / (batch32c_ms * 1e-3) / 1e9, 4),
                "speedup_vs_sequential_plain_fp32": round(seq_ms / batch32c_ms, 3),
                "rel_err_vs_fp64": err32c},
            "f16_compensated_batch": {
                "ms_per_step": round(batch16_ms, 3),
                "value": round(n_total * world / (batch16_ms * 1e-3) / 1e9, 4),
                "speedup_vs_sequential_plain_fp32": round(seq_ms / batch16_ms, 3),
                "rel_err_vs_fp64": err16,
                "note": "FP16 kernel cubes quantise the kernel values to "
                        "about 1e-4 relative, above the 1e-5 bar: a "
                        "1e-4 mode"},
            "f16_compensated_central_batch": {
                "ms_per_step": round(batch16c_ms, 3),
                "value": round(n_total * world / (batch16c_ms * 1e-3) / 1e9, 4),
                "speedup_vs_sequential_plain_fp32": round(seq_ms / batch16c_ms, 3),
                "rel_err_vs_fp64": err16c},
            "clocks": clk}


def central_radius(chans, frac):
    """Chebyshev distance from the grid centre, in cells, within which
    `frac` of all channels' visibilities lie."""
    d = []
    for c in chans:
        sc = c.grid_size * float(np.float32(c.cell_size_rad))
        d.append(torch.maximum(c.uu.abs(), c.vv.abs()).float() * sc)
    d = torch.cat(d)
    k = max(1, int(frac * d.numel()))
    return int(math.ceil(float(torch.kthvalue(d, k).values))) + 1


def audit_batch(chans, cubes, ws, opts, m=100000):
    """Relative RMS vs the FP64 oracle of the batched path (cubes and
    options as timed) on seeded samples of the lowest and highest
    channel."""
    import fpga_gridding_b200 as fg
    from fpga_gridding_b200 import _lib
    O = ensure_oracle()
    out = {}
    for idx in (0, len(chans) - 1):
        c = chans[idx]
        rng = np.random.default_rng(11 + idx)
        sel = torch.as_tensor(np.sort(rng.choice(c.num_points,
                                                 size=min(m, c.num_points),
                                                 replace=False)),
                              device=c.uu.device)
        sub = c.subset(sel)
        hd = host_dict(sub)
        sd = dict(hd)
        for k in ("conv_func", "uu", "vv", "ww", "vis", "weight"):
            sd[k] = np.asarray(hd[k], np.float64)
        _, n_ref, g_ref = O.grid_d(sd, threads=host_threads())
        grid = torch.zeros(2 * c.grid_size ** 2, device="cuda")
        norm = torch.zeros(1, dtype=torch.float64, device="cuda")
        fg.grid_batch_device(ws, [dict(
            cube=cubes[idx], uu=sub.uu, vv=sub.vv, ww=sub.ww, vis=sub.vis,
            weight=sub.weight, cell_size_rad=hd["cell_size_rad"],
            w_scale=hd["w_scale"], grid_size=c.grid_size, grid=grid,
            d_norm=norm)], opts=opts)
        torch.cuda.synchronize()
        out[f"channel_{idx}"] = {
            "grid_rel_rms": O.rel_rms(grid.cpu().numpy(), g_ref),
            "norm_rel": abs(norm.item() - n_ref) / abs(n_ref),
            "sample": f"{len(sel)} seeded visibilities"}
    return out


SERVING_DESC = ("serving: 2000 jobs, visibilities log-uniform in 1e4-5e7, "
                "grids {512,1024,2048,4096,8192}^2 FP32, 8-256 w-planes, "
                "support 3-32, {kt} kernel cubes (20% shared), seeded Poisson "
                "arrivals at 70% of measured capacity, 150 GB HBM budget")


def run_serving(args, world, rank, local):
    """Resident server under a Poisson stream: jobs/s, p50/p99 latency,
    isolated-job latency, and an audit of 5% of the jobs (mix vs alone, and
    the FP64 oracle where the job is small enough)."""
    import fpga_gridding_b200 as fg
    from fpga_gridding_b200 import _lib, workloads as W
    from fpga_gridding_b200.serving import Server

    num_jobs = args.serving_jobs
    base, jobs, specs = W.serving_stream(num_jobs=num_jobs,
                                         seed=4 + rank + args.serving_seed,
                                         device="cuda")
    ws = fg.Workspace(local)
    cubes = {}
    f16 = args.serving_kernel == "f16"
    for key, (sup, csh) in specs.items():
        cube = W.analytic_kernel_cube(sup, 4, csh, device="cuda").float()
        cubes[key] = fg.Cube(ws, sup, 4, csh, cube, data_is_double=False,
                             kernel_type=_lib.KERNEL_F16 if f16
                             else _lib.KERNEL_NATIVE)
        del cube
    torch.cuda.synchronize()
    srv = Server(local, budget_bytes=150 << 30, slots=args.serving_slots,
                 max_batch=args.serving_batch)

    def submit(i):
        j = jobs[i]
        s, e = j["start"], j["start"] + j["n"]
        srv.submit(i, cubes[j["cube_key"]], base["uu"][s:e], base["vv"][s:e],
                   base["ww"][s:e], base["vis"][2 * s:2 * e],
                   base["weight"][s:e], j["cell_size_rad"], j["w_scale"],
                   j["grid_size"])

    rng = np.random.default_rng(123 + rank + args.serving_seed)
    audited = set(rng.choice(num_jobs, size=max(1, num_jobs // 20),
                             replace=False).tolist())
    alone_grids = {}

    def drain(pending, keep=None):
        out = {}
        while pending:
            for c in srv.poll(timeout=1.0):
                if c["status"] != 0:
                    raise RuntimeError(f"job {c['tag']} status {c['status']}")
                if keep is not None and c["tag"] in keep:
                    keep[c["tag"]] = srv.grid(c).cpu().numpy()
                srv.release(c["tag"])
                out[c["tag"]] = c
                pending.discard(c["tag"])
        return out

    # warm-up: the largest jobs, several at once, so that every slot's
    # workspace reaches its working size before anything is timed
    big = sorted(range(num_jobs), key=lambda i: -jobs[i]["n"])
    for _ in range(2):
        warm = set(big[:4 * args.serving_slots])
        for i in warm:
            submit(i)
        drain(set(warm))
    # isolated latency: one job at a time.  Their sum is the time the
    # server needs for the stream without any batching or overlap: its
    # inverse is the capacity the arrival rate is set against.
    iso = {}
    for i in range(num_jobs):
        submit(i)
        keep = {i: None} if i in audited else None
        c = drain({i}, keep)[i]
        iso[i] = c["end_s"] - c["submit_s"]
        if keep:
            alone_grids[i] = keep[i]
    capacity = num_jobs / sum(iso.values())
    # burst throughput: every job submitted at once (maximal batching)
    t0 = srv.clock()
    for i in range(num_jobs):
        submit(i)
    done = drain(set(range(num_jobs)))
    burst = num_jobs / (max(c["end_s"] for c in done.values()) - t0)
    # Poisson arrivals at 70% of capacity
    rate = args.serving_rate if args.serving_rate > 0 else 0.7 * capacity
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=num_jobs))
    mix_grids = {i: None for i in audited}
    lat, waits, batch_sizes, mem_peak = {}, {}, [], 0
    start = srv.clock()
    nxt = 0
    pending = set()
    while nxt < num_jobs or pending:
        now = srv.clock() - start
        while nxt < num_jobs and arrivals[nxt] <= now:
            submit(nxt)
            pending.add(nxt)
            nxt += 1
        wait = max(0.0, arrivals[nxt] - (srv.clock() - start)) if nxt < num_jobs else 0.5
        for c in srv.poll(timeout=min(wait, 0.5)):
            if c["status"] != 0:
                raise RuntimeError(f"job {c['tag']} status {c['status']}")
            lat[c["tag"]] = c["end_s"] - c["submit_s"]
            waits[c["tag"]] = c["start_s"] - c["submit_s"]
            batch_sizes.append(c["batch_size"])
            if c["tag"] in mix_grids:
                # read after the stream (a copy here would hold up arrivals)
                mix_grids[c["tag"]] = c
            else:
                srv.release(c["tag"])
            pending.discard(c["tag"])
        mem_peak = max(mem_peak, srv.memory()[0])
    span = srv.clock() - start
    for i, c in mix_grids.items():
        mix_grids[i] = srv.grid(c).cpu().numpy()
        srv.release(i)
    srv.close()
    lat_v = np.array([lat[i] for i in range(num_jobs)])
    iso_v = np.array([iso[i] for i in range(num_jobs)])
    ratio = lat_v / iso_v
    # the jobs at or above the p99 latency: how long they queued for a slot
    # and how long they ran, against their isolated latency
    top = [i for i in range(num_jobs) if lat[i] >= np.percentile(lat_v, 99)]
    tail = {"jobs": len(top),
            "mean_visibilities": float(np.mean([jobs[i]["n"] for i in top])),
            "mean_queue_s": float(np.mean([waits[i] for i in top])),
            "mean_run_s": float(np.mean([lat[i] - waits[i] for i in top])),
            "mean_isolated_s": float(np.mean([iso[i] for i in top]))}
    points = sum(j["n"] for j in jobs)

    # audit: mix vs alone for 5% of the jobs, FP64 oracle for the small ones
    from oracle.oracle import rel_rms
    same = [rel_rms(mix_grids[i], alone_grids[i]) for i in sorted(audited)]
    oracle_err = []
    if not args.no_cpu_baseline:
        O = ensure_oracle()
        for i in sorted(audited):
            j = jobs[i]
            if j["n"] > 300000:
                continue
            s, e = j["start"], j["start"] + j["n"]
            sup, csh = specs[j["cube_key"]]
            d = dict(num_w_planes=len(sup), support=sup, oversample=4,
                     conv_size_half=csh,
                     conv_func=W.analytic_kernel_cube(sup, 4, csh).float()
                     .double().numpy(),
                     uu=base["uu"][s:e].double().cpu().numpy(),
                     vv=base["vv"][s:e].double().cpu().numpy(),
                     ww=base["ww"][s:e].double().cpu().numpy(),
                     vis=base["vis"][2 * s:2 * e].double().cpu().numpy(),
                     weight=np.ones(j["n"]), cell_size_rad=j["cell_size_rad"],
                     w_scale=j["w_scale"], grid_size=j["grid_size"])
            _, _, ref = O.grid_d(d, threads=host_threads())
            oracle_err.append(rel_rms(alone_grids[i], ref))
    for c in cubes.values():
        c.close()
    ws.close()
    pct = lambda a, q: float(np.percentile(a, q))
    return {"metric": METRIC, "value": round(points / span / 1e9, 4),
            "unit": UNIT, "n_gpus": world, "steps": num_jobs, "warmup": 16,
            "ms_per_step": round(1e3 * span / num_jobs, 3),
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f16 kernels, f32" if f16 else "f32", "data": DATA_DESC,
            "config": {"workload": SERVING_DESC.replace(
                           "{kt}", "FP16" if f16 else "FP32"), "jobs": num_jobs,
                       "seed": args.serving_seed,
                       "points": points, "slots": args.serving_slots,
                       "max_batch": args.serving_batch},
            "capacity_jobs_per_s": capacity,
            "capacity_definition": "jobs / sum of isolated (one at a time) "
                                   "latencies: the service rate without "
                                   "batching or overlap",
            "burst_jobs_per_s": burst,
            "offered_jobs_per_s": rate,
            "achieved_jobs_per_s": num_jobs / span,
            "latency_s": {"p50": pct(lat_v, 50), "p99": pct(lat_v, 99)},
            "isolated_latency_s": {"p50": pct(iso_v, 50), "p99": pct(iso_v, 99)},
            "slowdown_vs_isolated": {"p50": pct(ratio, 50),
                                     "p99": pct(ratio, 99)},
            "p99_latency_over_p99_isolated": pct(lat_v, 99) / pct(iso_v, 99),
            "p99_tail": tail,
            "mean_batch_size": float(np.mean(batch_sizes)),
            "server_memory_peak_bytes": mem_peak,
            "audit": {"jobs": len(audited),
                      "mix_vs_alone_rel_rms_max": max(same) if same else None,
                      "fp64_oracle_rel_rms_max": max(oracle_err) if oracle_err else None,
                      "fp64_oracle_jobs": len(oracle_err)}}


WEIGHTS_DESC = ("weights: one uniform-weighting pass (weights-grid write, "
                "then density read: oskar_grid_weights_write_f / _read_f) "
                "over plain_large's 39,244,800 uv points with unit weights "
                "(as main.cpp:203); 8192^2 FP32 weights grid, zero-filled "
                "each pass; float coordinate arithmetic")


def weights_threads(grid_size):
    """Host threads for the weights CPU baseline: all of them, bounded by
    memory for the private FP32 weights grids."""
    grid_bytes = grid_size * grid_size * 4
    t = host_threads()
    return max(1, min(t, int(0.4 * mem_available_bytes() // grid_bytes), 256))


def run_weights(args, world, rank, local):
    """Uniform weighting on the GPU: ordered (bit-exact for any weights)
    write + read per step; the atomic write is timed beside it."""
    import fpga_gridding_b200 as fg
    wl = make_workload(rank, args.stations)
    n = wl.num_points
    g = wl.grid_size
    cell = float(np.float32(wl.cell_size_rad))
    ws = fg.Workspace(local)
    s = torch.cuda.Stream()
    wgrid = torch.zeros(g * g, dtype=torch.float32, device="cuda")
    wout = torch.zeros(n, dtype=torch.float32, device="cuda")
    sk_w = torch.zeros(1, dtype=torch.int64, device="cuda")
    sk_r = torch.zeros(1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()

    def step(ordered):
        with torch.cuda.stream(s):
            wgrid.zero_()
        fg.weights_write_device(ws, wl.uu, wl.vv, wl.weight, cell, g, wgrid,
                                sk_w, ordered=ordered, stream=s)
        fg.weights_read_device(ws, wl.uu, wl.vv, wl.weight, wout, cell, g,
                               wgrid, sk_r, stream=s)

    def timed(ordered):
        for _ in range(args.warmup):
            step(ordered)
        s.synchronize()
        barrier(world)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(args.steps):
            step(ordered)
        e1.record(s)
        e1.synchronize()
        return max_over_ranks(e0.elapsed_time(e1) / args.steps, world)

    # kernels of one pass: the write's (from the workspace statistics), the
    # read's one kernel; the zero fill is torch's
    fg.weights_write_device(ws, wl.uu, wl.vv, wl.weight, cell, g, wgrid,
                            sk_w, ordered=True, stream=s)
    s.synchronize()
    launches_write = ws.stats().kernel_launches
    wgrid.zero_()
    clocks = ClockSampler(local)
    clocks.start()
    ordered_ms = timed(True)
    clk = clocks.stop()
    g_ord = wgrid.cpu().numpy()
    w_ord = wout.cpu().numpy()
    skips = (int(sk_w.item()), int(sk_r.item()))
    atomic_ms = timed(False)
    g_atm = wgrid.cpu().numpy()
    w_atm = wout.cpu().numpy()
    value = n * world / (ordered_ms * 1e-3) / 1e9
    alg_bytes = 28 * n + 16 * g * g
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (ordered_ms * 1e-3) / 1e9
    achieved_atm = alg_bytes / (atomic_ms * 1e-3) / 1e9
    out = {"metric": "uniform-weighting throughput (weights write + read)",
           "value": round(value, 4), "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(ordered_ms, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": DATA_DESC,
           "config": {"workload": WEIGHTS_DESC, "num_points": n,
                      "grid_size": g, "mode": "ordered write (stable sort "
                      "by cell, one sequential sum per cell) + read",
                      "l2": "inputs (0.6 GB/step) larger than L2; no flush"},
           "roofline": {"kernel": "whole pass (key, radix sort, run sum, "
                                  "read)", "bound": "hbm",
                        "achieved": round(achieved, 2), "peak": peak,
                        "peak_source": peak_kind, "unit": "GB/s",
                        "frac": round(achieved / peak, 4), "traffic": None,
                        "algorithmic_bytes_per_launch": alg_bytes},
           "atomic_pass": {"ms_per_step": round(atomic_ms, 3),
                           "value": round(n * world / (atomic_ms * 1e-3)
                                          / 1e9, 4),
                           "hbm_frac": round(achieved_atm / peak, 4),
                           "grid_equal_to_ordered": bool(
                               np.array_equal(g_atm, g_ord)),
                           "weights_equal_to_ordered": bool(
                               np.array_equal(w_atm, w_ord))},
           "gpu_launches": (launches_write + 1) * args.steps,
           "skipped": {"write": skips[0], "read": skips[1]},
           "clocks": clk}
    if not args.no_e2e:
        out["e2e"] = run_weights_e2e(args, wl, world)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        O = ensure_oracle()
        use_ref = O.reference_lib() is not None
        hd = host_dict(wl)
        rsk_w, rg, rsk_r, rw, (tw, tr) = O.weights_timed(
            hd["uu"], hd["vv"], hd["weight"], hd["cell_size_rad"], g,
            np.zeros(g * g, np.float32), np.zeros(n, np.float32),
            single=True, use_reference=use_ref)
        kind = "reference" if use_ref else "port"
        t = weights_threads(g)
        secs, _, _, _, _ = O.time_weights_parallel(
            hd["uu"], hd["vv"], hd["weight"], hd["cell_size_rad"], g, t,
            use_ref)
        out["cpu_baseline"] = {
            "value": round(n / secs / 1e9, 6), "unit": UNIT, "cores": t,
            "kind": kind,
            "serial_value": round(n / (tw + tr) / 1e9, 6),
            "sample": f"the whole workload, once: {'reference' if use_ref else 'restated'} "
                      f"oskar_grid_weights_write_f on {t} threads with "
                      f"private grids over slices, a parallel sum of the "
                      f"grids, then _read_f over slices; {secs:.3f} s "
                      f"(serial_value: one thread, {tw + tr:.3f} s)"}
        out["parity_vs_reference"] = {
            "skipped_equal": (rsk_w, rsk_r) == skips,
            "grid_bit_exact": bool(np.array_equal(rg, g_ord)),
            "weights_bit_exact": bool(np.array_equal(rw, w_ord)),
            "atomic_grid_bit_exact": bool(np.array_equal(rg, g_atm)),
            "sample": "the whole workload"}
    return out


def run_weights_e2e(args, wl, world):
    """oskar_grid_weights_write_f then _read_f (drop-in C ABI) on pinned
    host buffers, K steps."""
    import fpga_gridding_b200 as fg
    pin = lambda t: t.cpu().pin_memory()
    h = {k: pin(getattr(wl, k)).numpy() for k in ("uu", "vv", "weight")}
    n = wl.num_points
    g = wl.grid_size
    hgrid = torch.zeros(g * g, dtype=torch.float32).pin_memory().numpy()
    hout = torch.zeros(n, dtype=torch.float32).pin_memory().numpy()
    cell = float(np.float32(wl.cell_size_rad))

    def call():
        fg.oskar_grid_weights_write_f(n, h["uu"], h["vv"], h["weight"], cell,
                                      g, hgrid)
        fg.oskar_grid_weights_read_f(n, h["uu"], h["vv"], h["weight"], hout,
                                     cell, g, hgrid)
    for _ in range(max(1, args.warmup)):
        hgrid[:] = 0.0
        call()
    barrier(world)
    secs = 0.0
    for _ in range(args.steps):
        # the caller's grid starts at zero each step (main.cpp:208 allocates
        # it zeroed once); filling it is the caller's work, not timed
        hgrid[:] = 0.0
        t0 = time.perf_counter()
        call()
        secs += time.perf_counter() - t0
    secs = max_over_ranks(secs, world)
    fg.load().oskar_grid_wproj_b200_release_thread_cache()
    return {"value": round(n * args.steps * world / secs / 1e9, 4),
            "unit": UNIT,
            "h2d_bytes_per_step": n * 12 + n * 16 + 2 * g * g * 4,
            "d2h_bytes_per_step": g * g * 4 + n * 4 + 16,
            "ms_per_step": round(1e3 * secs / args.steps, 3),
            "path": "oskar_grid_weights_write_f + _read_f (drop-in C ABI), "
                    "pinned host buffers; the caller's zero fill of the "
                    "weights grid before each step is outside the timed "
                    "region"}


def run_reference_weights(args, world):
    """Reference arm of the weights workload: the reference's serial
    oskar_grid_weights_write_f + _read_f over the whole workload per step."""
    O = ensure_oracle()
    use_ref = O.reference_lib() is not None
    wl = make_workload(0)
    hd = host_dict(wl)
    n = len(hd["uu"])
    g = hd["grid_size"]
    del wl
    t = weights_threads(g)
    tot = 0.0
    for i in range(args.warmup + args.steps):
        secs, _, _, _, _ = O.time_weights_parallel(
            hd["uu"], hd["vv"], hd["weight"], hd["cell_size_rad"], g, t,
            use_ref)
        if i >= args.warmup:
            tot += secs
    value = n * args.steps / tot / 1e9
    kind = "reference" if use_ref else "port"
    return {"impl": "reference",
            "metric": "uniform-weighting throughput (weights write + read)",
            "value": round(value, 6), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * tot / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": DATA_DESC,
            "config": {"workload": WEIGHTS_DESC, "num_points": n,
                       "grid_size": g},
            "cpu_baseline": {"value": round(value, 6), "unit": UNIT,
                             "cores": t, "kind": kind,
                             "sample": f"each step: the whole workload; "
                                       f"oskar_grid_weights_write_f on {t} "
                                       f"threads with private grids over "
                                       f"slices, a parallel sum of the "
                                       f"grids, then _read_f over slices"},
            "e2e": {"value": round(value, 6), "unit": UNIT,
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


DEGRID_DESC = ("degrid: the adjoint of plain_large's gridding - its "
               "39,244,800 visibilities predicted from a seeded random "
               "8192^2 complex64 grid with the same 256 w-planes (support "
               "4->36, oversample 4); FP32, FP64 coordinates")


def _degrid_cpu(O, hd, grid64, threads, m):
    """The oracle's degridder (FP64; the reference has none) on a seeded
    sample of m visibilities, split over `threads` host threads (ctypes
    releases the GIL).  Returns (seconds, sample indices, vis)."""
    from concurrent.futures import ThreadPoolExecutor
    rng = np.random.default_rng(21)
    idx = np.sort(rng.choice(len(hd["uu"]), size=m, replace=False))
    sub = dict(hd)
    for k in ("uu", "vv", "ww", "weight"):
        sub[k] = np.asarray(hd[k][idx], np.float64)
    sub["conv_func"] = np.asarray(hd["conv_func"], np.float64)
    edges = np.linspace(0, m, threads + 1).astype(int)
    parts = []
    for a, b in zip(edges[:-1], edges[1:]):
        p = dict(sub)
        for k in ("uu", "vv", "ww", "weight"):
            p[k] = sub[k][a:b]
        p["vis"] = np.zeros(2 * (b - a))
        parts.append(p)
    t0 = time.perf_counter()
    with ThreadPoolExecutor(threads) as ex:
        res = list(ex.map(lambda p: O.degrid_d(p, grid64), parts))
    secs = time.perf_counter() - t0
    vis = np.concatenate([r[1] for r in res])
    return secs, idx, vis


def run_degrid(args, world, rank, local):
    """Degridding (oskar_b200_degrid) at plain_large size."""
    import fpga_gridding_b200 as fg
    lib = fg.load()
    wl = make_workload(rank, args.stations)
    n = wl.num_points
    g = wl.grid_size
    cell = float(np.float32(wl.cell_size_rad))
    wsc = float(np.float32(wl.w_scale))
    ws = fg.Workspace(local)
    cube = fg.Cube(ws, wl.support, wl.oversample, wl.conv_size_half,
                   wl.conv_func, data_is_double=False)
    gen = torch.Generator(device="cuda").manual_seed(17 + rank)
    grid = torch.randn(2 * g * g, generator=gen, device="cuda")
    vis = torch.zeros(2 * n, device="cuda")
    skip = torch.zeros(1, dtype=torch.int64, device="cuda")
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    lib.oskar_b200_set_stage_timing(ws.handle, 1)

    def step():
        fg.degrid_device(ws, cube, wl.uu, wl.vv, wl.ww, wl.weight, cell, wsc,
                         g, grid, vis, skip, stream=s)

    for _ in range(args.warmup):
        step()
    s.synchronize()
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    kern_ms, launches = [], 0
    e0.record(s)
    for _ in range(args.steps):
        step()
        s.synchronize()   # this step's stage events are now readable
        st = ws.stats()
        kern_ms.append(st.grid_ms)
        launches += st.kernel_launches
    e1.record(s)
    e1.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    taps = st.grid_updates
    kernel_ms = statistics.mean(kern_ms)
    # per visibility: 16-byte record, 4-byte order value, 4-byte key, 8-byte
    # result; plus the grid read once and the kernel slabs
    alg = n * (16 + 4 + 4 + 8) + g * g * 8 + cube.bytes
    peak, peak_kind = measured_peaks()
    achieved = alg / (kernel_ms * 1e-3) / 1e9
    out = {"metric": "degridding throughput (visibilities predicted)",
           "value": round(n * world / (ms * 1e-3) / 1e9, 4), "unit": UNIT,
           "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(ms, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": DATA_DESC,
           "config": {"workload": DEGRID_DESC, "num_points": n,
                      "grid_size": g,
                      "l2": "inputs and grid (1.0 GB/step) larger than L2; "
                            "no flush"},
           "kernel_taps_per_s": taps / (kernel_ms * 1e-3),
           "stage_ms": {"prep": round(st.prep_ms, 3),
                        "sort": round(st.sort_ms, 3),
                        "degrid": round(st.grid_ms, 3)},
           "roofline": {"kernel": "degrid_kernel<float,float2>",
                        "bound": "issue",
                        "bound_evidence": "ncu: L1 loads of kernel values "
                                          "and grid cells and instruction "
                                          "issue limit it; DRAM throughput "
                                          "about 5 %",
                        "achieved": round(achieved, 2),
                        "peak": peak, "peak_source": peak_kind,
                        "unit": "GB/s", "frac": round(achieved / peak, 4),
                        "traffic": profiled_value(
                            "dram_bytes_per_launch_full_job",
                            "degrid_kernel_plain_large.md"),
                        "traffic_source": "ncu dram__bytes_read.sum + "
                                          "dram__bytes_write.sum of one "
                                          "full-size launch, copied from "
                                          "profiles/degrid_kernel_plain_"
                                          "large.md (not measured in this "
                                          "run)",
                        "algorithmic_bytes_per_launch": alg,
                        "kernel_ms": round(kernel_ms, 3)},
           "gpu_launches": launches, "skipped": int(skip.item()),
           "clocks": clk}
    if not args.no_e2e:
        # Host buffers (pinned): the C-ABI call oskar_b200_degrid_host
        # uploads the grid, then the coordinates (and current values) of the
        # visibilities in chunks, degrids each chunk as it lands and copies
        # its predictions back while later chunks upload.
        pin = lambda t: t.cpu().pin_memory().numpy()
        h = {k: pin(getattr(wl, k)) for k in ("uu", "vv", "ww")}
        hg = pin(grid)
        hv = pin(torch.zeros(2 * n, dtype=torch.float32))
        secs = []
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            fg.degrid_host(ws, cube, h["uu"], h["vv"], h["ww"], None, cell,
                           wsc, g, hg, hv)
            if i >= args.warmup:
                secs.append(time.perf_counter() - t0)
        ems = max_over_ranks(1e3 * sum(secs) / len(secs), world)
        out["e2e"] = {"value": round(n * world / (ems * 1e-3) / 1e9, 4),
                      "unit": UNIT, "h2d_bytes_per_step": n * 20 + g * g * 8,
                      "d2h_bytes_per_step": n * 8,
                      "ms_per_step": round(ems, 3),
                      "path": "oskar_b200_degrid_host (C ABI) on pinned host "
                              "arrays: grid and coordinates up, "
                              "visibilities down, copies overlapped with "
                              "the degridding"}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        O = ensure_oracle()
        hd = host_dict(wl)
        g64 = grid.double().cpu().numpy()
        t = host_threads()
        # calibrate, then about cpu_seconds of work
        secs, idx, _ = _degrid_cpu(O, hd, g64, t, 20000 * t)
        m = int(min(n, max(20000 * t, 20000 * t / secs * args.cpu_seconds)))
        secs, idx, cpu_vis = _degrid_cpu(O, hd, g64, t, m)
        gpu_vis = vis.double().cpu().numpy().reshape(-1, 2)[idx].reshape(-1)
        out["cpu_baseline"] = {
            "value": round(m / secs / 1e9, 6), "unit": UNIT, "cores": t,
            "kind": "port",
            "sample": f"{m} seeded visibilities of the workload; the "
                      f"oracle's FP64 degridder (the reference has none) on "
                      f"{t} threads over slices; {secs:.2f} s"}
        out["rel_err_vs_fp64"] = {
            "vis_rel_rms": O.rel_rms(gpu_vis, cpu_vis),
            "sample": f"the same {m} visibilities, FP32 GPU vs FP64 oracle "
                      f"on the same float inputs and grid"}
    cube.close()
    return out


PRECISION_DESC = ("precision: 512 stations uniform in a 5 km disk x 3000 "
                  "samples at 150 MHz (392,448,000 visibilities concentrated "
                  "near the uv origin); grid 4096^2; 128 w-planes, support "
                  "4->32, oversample 8; FP32 inputs (FP64 mode: the same "
                  "values promoted)")


def run_precision(args, world, rank, local):
    """The grid-precision modes on one long-integration job: speed of each
    at full size, error of each against the FP64 GPU grid at full size and
    against the CPU FP64 oracle on a seeded sample."""
    import fpga_gridding_b200 as fg
    from fpga_gridding_b200 import _lib, workloads as W
    O = ensure_oracle()
    num_times = 3000 if args.stations == 512 else 300
    wl = W.precision_sweep(seed=3 + rank, device="cuda",
                           num_stations=args.stations,
                           num_times=num_times).to(dtype=torch.float32)
    torch.cuda.empty_cache()
    n, g = wl.num_points, wl.grid_size
    cell = float(np.float32(wl.cell_size_rad))
    wsc = float(np.float32(wl.w_scale))
    ws = fg.Workspace(local)
    lib = fg.load()
    s = torch.cuda.Stream()
    modes = [("fp32", False, _lib.KERNEL_NATIVE, _lib.ACCUM_PLAIN),
             ("f16", False, _lib.KERNEL_F16, _lib.ACCUM_PLAIN),
             ("bf16", False, _lib.KERNEL_BF16, _lib.ACCUM_PLAIN),
             ("f16_compensated", False, _lib.KERNEL_F16,
              _lib.ACCUM_COMPENSATED),
             ("fp32_compensated", False, _lib.KERNEL_NATIVE,
              _lib.ACCUM_COMPENSATED),
             ("fp64", True, _lib.KERNEL_NATIVE, _lib.ACCUM_PLAIN)]
    rng = np.random.default_rng(31)
    m = min(n, 200000)
    sel = torch.as_tensor(np.sort(rng.choice(n, size=m, replace=False)),
                          device="cuda")
    sub = wl.subset(sel)
    hd = host_dict(sub)
    ref_sample = dict(hd)
    for k in ("conv_func", "uu", "vv", "ww", "vis", "weight"):
        ref_sample[k] = np.asarray(hd[k], np.float64)
    _, _, g_oracle = O.grid_d(ref_sample, threads=host_threads())
    results, grids = {}, {}
    for name, dbl, kt, acc in modes:
        real = torch.float64 if dbl else torch.float32
        conv = wl.conv_func.double() if dbl else wl.conv_func
        cube = fg.Cube(ws, wl.support, wl.oversample, wl.conv_size_half, conv,
                       data_is_double=dbl, kernel_type=kt)
        inp = [t.to(real) for t in (wl.uu, wl.vv, wl.ww, wl.vis, wl.weight)]
        grid = torch.zeros(2 * g * g, dtype=real, device="cuda")
        opts = fg.options(accum_mode=acc)

        def step():
            fg.grid_device(ws, cube, *inp, cell, wsc, g, grid, opts=opts,
                           stream=s)
        for _ in range(args.warmup):
            step()
        s.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(args.steps):
            step()
        e1.record(s)
        e1.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
        grid.zero_()
        step()
        s.synchronize()
        grids[name] = grid.double()
        # the audited sample through the same mode
        sg = torch.zeros(2 * g * g, dtype=real, device="cuda")
        fg.grid_device(ws, cube, *[t.to(real) for t in
                                   (sub.uu, sub.vv, sub.ww, sub.vis,
                                    sub.weight)],
                       cell, wsc, g, sg, opts=opts, stream=s)
        s.synchronize()
        results[name] = {
            "ms_per_step": round(ms, 3),
            "gvis_per_s": round(n * world / (ms * 1e-3) / 1e9, 4),
            "rel_rms_vs_cpu_fp64_oracle_sample": O.rel_rms(
                sg.double().cpu().numpy(), g_oracle)}
        del inp, grid, sg
        cube.close()
        torch.cuda.empty_cache()
    ref = grids["fp64"]
    for name in results:
        d = grids[name] - ref
        results[name]["rel_rms_vs_fp64_full"] = float(
            torch.sqrt((d * d).sum() / (ref * ref).sum()).item())
        results[name]["max_cell_err_rel_to_max_cell"] = float(
            (d.abs().max() / ref.abs().max()).item())
    fp32 = results["fp32"]
    return {"metric": METRIC, "value": fp32["gvis_per_s"], "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": fp32["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": DATA_DESC,
            "config": {"workload": PRECISION_DESC if args.stations == 512
                       else f"profiling case: {args.stations} stations x "
                            f"{num_times} samples, otherwise as precision",
                       "num_points": n, "grid_size": g,
                       "l2": "inputs (9.4 GB/step) larger than L2; no flush"},
            "modes": results,
            "error_note": "rel_rms_vs_fp64_full: each mode's full-size grid "
                          "against the GPU FP64 grid of the same inputs; "
                          "rel_rms_vs_cpu_fp64_oracle_sample: a seeded "
                          f"{m}-visibility sample gridded by each mode "
                          "against the CPU FP64 oracle (bit-identical to the "
                          "reference's oskar_grid_wproj_d)"}


def run_reference(args, world, rank):
    if rank != 0:
        return None
    if args.workload == "weights":
        return run_reference_weights(args, world)
    if args.workload == "degrid":
        return {"impl": "reference",
                "unavailable": "the reference has no degridder (Defines.h:48 "
                               "only reserves a DEGRIDDING switch)"}
    if args.workload in ("batch128", "serving", "precision"):
        return {"impl": "reference",
                "unavailable": f"the reference has no {args.workload} path; "
                               "its gridder is timed by the default workload"}
    O = ensure_oracle()
    use_ref = O.reference_lib() is not None
    wl = make_workload(0)
    hd = host_dict(wl)
    config = plain_config(512, wl.num_points, wl.grid_size, wl.num_w_planes,
                          wl.oversample, world)
    del wl
    torch.cuda.empty_cache() if torch.cuda.is_available() else None
    per_step_s = max(2.0, min(10.0, 120.0 / max(1, args.steps + args.warmup)))
    tot_secs, tot_m, tot_taps, t, kind = 0.0, 0, 0, 1, "port"
    for i in range(args.warmup + args.steps):
        secs, m, taps, t, kind = cpu_sample_time(O, hd, True, use_ref,
                                                 per_step_s, seed=1000 + i)
        if i >= args.warmup:
            tot_secs += secs
            tot_m += m
            tot_taps += taps
    value = tot_m / tot_secs / 1e9
    desc = ("reference oskar_grid_wproj_f (oskar_grid_wproj.c compiled "
            "unmodified), driven in its fixed 10000-point calls"
            if kind == "reference" else "C restatement of oskar_grid_wproj_f")
    return {"impl": "reference", "metric": METRIC, "value": round(value, 6),
            "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(1e3 * tot_secs / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": DATA_DESC,
            "config": config,
            "grid_updates_per_s": tot_taps / tot_secs,
            "cpu_baseline": {"value": round(value, 6), "unit": UNIT,
                             "cores": t, "kind": kind,
                             "sample": f"each step: about {per_step_s:.0f} s "
                                       f"of a seeded uniform sample of the "
                                       f"workload's visibilities; {desc}; "
                                       f"{t} threads with private grids"},
            "e2e": {"value": round(value, 6), "unit": UNIT,
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--cpu-seconds", type=float, default=8.0,
                    help="target wall time of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", choices=("plain_large", "batch128",
                                           "serving", "weights", "degrid",
                                           "precision"),
                    default="plain_large",
                    help="plain_large (the benchmark job), batch128 (the "
                         "128-channel batching workload), serving (the "
                         "Poisson job stream) or weights (uniform "
                         "weighting over the benchmark job's uv points)")
    ap.add_argument("--autotune", action="store_true",
                    help="measure classes per thread per support on a "
                         "sample of the job before timing")
    ap.add_argument("--cpt", type=int, default=0,
                    help="gridding classes per thread for every support "
                         "(0: the tuned table)")
    ap.add_argument("--serving-jobs", type=int, default=2000)
    ap.add_argument("--serving-rate", type=float, default=0.0,
                    help="serving arrival rate in jobs/s (default: 70%% of "
                         "the measured capacity)")
    ap.add_argument("--serving-slots", type=int, default=4,
                    help="concurrent batches the server keeps on the GPU")
    ap.add_argument("--serving-batch", type=int, default=32,
                    help="most jobs the server puts in one batch")
    ap.add_argument("--serving-seed", type=int, default=0,
                    help="offset of the serving stream's seeds (job mix, "
                         "arrivals, audited jobs)")
    ap.add_argument("--serving-kernel", choices=("f32", "f16"),
                    default="f32",
                    help="kernel-cube storage of the serving jobs (FP16 "
                         "quantises kernel values to ~1e-4 relative, above "
                         "the 1e-5 bar)")
    ap.add_argument("--stations", type=int, default=512,
                    help="stations of the job (512 = the benchmark job; "
                         "fewer = a smaller profiling case)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        # CPU only: rank 0 runs, the other ranks exit without work.
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        out = run_reference(args, world, rank)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.workload == "batch128":
            out = run_batch128(args, world, rank, local)
        elif args.workload == "serving":
            out = run_serving(args, world, rank, local)
        elif args.workload == "weights":
            out = run_weights(args, world, rank, local)
        elif args.workload == "degrid":
            out = run_degrid(args, world, rank, local)
        elif args.workload == "precision":
            out = run_precision(args, world, rank, local)
        else:
            out = run_b200(args, world, rank, local)
        if rank == 0 and out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
