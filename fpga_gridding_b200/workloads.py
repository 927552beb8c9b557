"""Seeded synthetic W-projection workloads.

No public dataset exists for this gridder (the reference's own test data,
<root>.vis with <root>_KERNELS_REAL/IMAG.fits, is not distributed), so every
workload here is generated: a station layout, Earth-rotation-synthesis uvw
tracks in wavelengths, a point-source sky with complex Gaussian noise, and an
analytic W-kernel cube (Gaussian taper times a w-dependent quadratic phase,
unit-sum normalised) laid out exactly as the reference reads it
(utils/read_kernel.c:89-94 and main.cpp:197-201): conv_func[plane][iv][iu]
with interleaved (re, im), holding only the non-negative quadrant in
oversampled units.

Visibilities are ordered time-major, baseline-minor (index = t * nb + b), the
order of the reference's visibility blocks (main.cpp:413-441).

Every generator is torch-based and runs on CPU (tests) or on a GPU (bench);
all randomness comes from one seeded torch.Generator on the CPU so results
do not depend on the device.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np
import torch

C_LIGHT = 299792458.0
OMEGA_EARTH = 7.2921150e-5  # rad/s


@dataclass
class Workload:
    """One gridding job in the reference's argument convention."""

    name: str
    uu: torch.Tensor        # [N] wavelengths
    vv: torch.Tensor        # [N]
    ww: torch.Tensor        # [N]
    vis: torch.Tensor       # [2N] interleaved re, im
    weight: torch.Tensor    # [N] (the reference ignores it)
    support: np.ndarray     # int32 [P]
    oversample: int
    conv_size_half: int
    conv_func: torch.Tensor  # [P * csh * csh * 2] interleaved
    cell_size_rad: float
    w_scale: float
    grid_size: int
    meta: dict = field(default_factory=dict)

    @property
    def num_points(self) -> int:
        return int(self.uu.numel())

    @property
    def num_w_planes(self) -> int:
        return int(self.support.shape[0])

    def to(self, dtype=None, device=None) -> "Workload":
        def cv(t):
            return t.to(dtype=dtype or t.dtype, device=device or t.device)
        return replace(self, uu=cv(self.uu), vv=cv(self.vv), ww=cv(self.ww),
                       vis=cv(self.vis), weight=cv(self.weight),
                       conv_func=cv(self.conv_func))

    def subset(self, index) -> "Workload":
        """Visibilities `index` (tensor of indices or a slice)."""
        vis2 = self.vis.view(-1, 2)[index].reshape(-1)
        return replace(self, uu=self.uu[index], vv=self.vv[index],
                       ww=self.ww[index], vis=vis2, weight=self.weight[index])

    def numpy(self) -> dict:
        """Host numpy arrays keyed by the reference's argument names."""
        return dict(
            num_w_planes=self.num_w_planes, support=self.support,
            oversample=self.oversample, conv_size_half=self.conv_size_half,
            conv_func=self.conv_func.cpu().numpy(),
            uu=self.uu.cpu().numpy(), vv=self.vv.cpu().numpy(),
            ww=self.ww.cpu().numpy(), vis=self.vis.cpu().numpy(),
            weight=self.weight.cpu().numpy(),
            cell_size_rad=self.cell_size_rad, w_scale=self.w_scale,
            grid_size=self.grid_size)


# --------------------------------------------------------------------------
# Array layouts and uvw synthesis
# --------------------------------------------------------------------------

def stations_uniform_disk(n: int, radius_m: float, gen: torch.Generator):
    """n stations uniform in a disk (east, north, up) metres."""
    r = radius_m * torch.sqrt(torch.rand(n, generator=gen, dtype=torch.float64))
    a = 2 * math.pi * torch.rand(n, generator=gen, dtype=torch.float64)
    return torch.stack([r * torch.cos(a), r * torch.sin(a),
                        torch.zeros(n, dtype=torch.float64)], 1)


def stations_log_radial(n: int, r_min_m: float, r_max_m: float,
                        gen: torch.Generator):
    """n stations with log-uniform radius (dense core, sparse arms)."""
    lr = math.log(r_min_m) + (math.log(r_max_m) - math.log(r_min_m)) * \
        torch.rand(n, generator=gen, dtype=torch.float64)
    r = torch.exp(lr)
    a = 2 * math.pi * torch.rand(n, generator=gen, dtype=torch.float64)
    return torch.stack([r * torch.cos(a), r * torch.sin(a),
                        torch.zeros(n, dtype=torch.float64)], 1)


def baselines_xyz(enu: torch.Tensor, lat_rad: float) -> torch.Tensor:
    """Baseline vectors (i < j) in the equatorial XYZ frame, metres."""
    e, nn, up = enu[:, 0], enu[:, 1], enu[:, 2]
    x = -math.sin(lat_rad) * nn + math.cos(lat_rad) * up
    y = e
    z = math.cos(lat_rad) * nn + math.sin(lat_rad) * up
    xyz = torch.stack([x, y, z], 1)
    i, j = torch.triu_indices(enu.shape[0], enu.shape[0], 1)
    return xyz[j] - xyz[i]


def earth_rotation_uvw(bxyz: torch.Tensor, num_times: int, dt_s: float,
                       freq_hz: float, dec_rad: float, device="cpu"):
    """uvw in wavelengths, time-major: index = t * num_baselines + b."""
    b = bxyz.to(device)
    t = torch.arange(num_times, dtype=torch.float64, device=device)
    ha = OMEGA_EARTH * dt_s * (t - 0.5 * (num_times - 1))  # centred on transit
    sh, ch = torch.sin(ha)[:, None], torch.cos(ha)[:, None]
    sd, cd = math.sin(dec_rad), math.cos(dec_rad)
    bx, by, bz = b[:, 0][None, :], b[:, 1][None, :], b[:, 2][None, :]
    scale = freq_hz / C_LIGHT
    u = (sh * bx + ch * by) * scale
    v = (-sd * ch * bx + sd * sh * by + cd * bz) * scale
    w = (cd * ch * bx - cd * sh * by + sd * bz) * scale
    return u.reshape(-1), v.reshape(-1), w.reshape(-1)


def point_source_vis(uu, vv, ww, num_sources: int, radius_rad: float,
                     noise_sigma: float, gen: torch.Generator,
                     chunk: int = 1 << 22):
    """Point sources of flux U(0.1, 1) Jy within radius_rad plus complex
    Gaussian noise; returns interleaved [2N] float64."""
    device = uu.device
    r = radius_rad * torch.sqrt(torch.rand(num_sources, generator=gen,
                                           dtype=torch.float64))
    a = 2 * math.pi * torch.rand(num_sources, generator=gen, dtype=torch.float64)
    l, m = r * torch.cos(a), r * torch.sin(a)
    n1 = torch.sqrt(1 - l * l - m * m) - 1
    flux = 0.1 + 0.9 * torch.rand(num_sources, generator=gen, dtype=torch.float64)
    l, m, n1, flux = (x.to(device) for x in (l, m, n1, flux))
    n_pts = uu.numel()
    noise = noise_sigma * torch.randn(2 * n_pts, generator=gen,
                                      dtype=torch.float64).to(device)
    out = torch.empty(n_pts, 2, dtype=torch.float64, device=device)
    for s in range(0, n_pts, chunk):
        e = min(n_pts, s + chunk)
        ph = -2 * math.pi * (uu[s:e, None] * l + vv[s:e, None] * m +
                             ww[s:e, None] * n1)
        out[s:e, 0] = (flux * torch.cos(ph)).sum(1)
        out[s:e, 1] = (flux * torch.sin(ph)).sum(1)
    return out.reshape(-1) + noise


# --------------------------------------------------------------------------
# Kernel cube
# --------------------------------------------------------------------------

def support_ramp(num_w_planes: int, s_min: int, s_max: int) -> np.ndarray:
    """Per-plane support, linear from s_min (plane 0) to s_max (last)."""
    if num_w_planes == 1:
        return np.array([s_min], dtype=np.int32)
    p = np.arange(num_w_planes, dtype=np.float64)
    return np.floor(s_min + (s_max - s_min) * p / (num_w_planes - 1) + 0.5
                    ).astype(np.int32)


def analytic_kernel_cube(support: np.ndarray, oversample: int,
                         conv_size_half: int, chirp: float = 0.02,
                         taper_div: float = 2.5, device="cpu"):
    """Gaussian taper exp(-r^2 / 2 sigma^2), sigma = support / taper_div
    cells, times phase exp(i 2 pi chirp p r^2), r = distance in grid cells;
    each plane scaled so its zero-offset taps sum to 1.  Returns the
    interleaved cube [P * csh * csh * 2] float64 (non-negative quadrant)."""
    num_planes = len(support)
    idx = torch.arange(conv_size_half, dtype=torch.float64, device=device)
    r2 = (idx[None, :] ** 2 + idx[:, None] ** 2) / float(oversample) ** 2
    s = torch.as_tensor(np.asarray(support, dtype=np.float64), device=device)
    sigma = s / taper_div
    taper = torch.exp(-r2[None] / (2 * (sigma * sigma)[:, None, None]))
    # zero-offset taps k = -S..S read quadrant index |k| * os: index 0 once,
    # k * os (k = 1..S) twice
    k = torch.arange(conv_size_half, device=device)
    on_tap = (k[None, :] % oversample == 0) & \
        (k[None, :] <= (s[:, None] * oversample))
    mult = on_tap.double() * torch.where(k[None, :] == 0, 1.0, 2.0)
    norm = torch.einsum("pi,pij,pj->p", mult, taper, mult)
    p = torch.arange(num_planes, dtype=torch.float64, device=device)
    phase = 2 * math.pi * chirp * p[:, None, None] * r2[None]
    cube = torch.stack([taper * torch.cos(phase), taper * torch.sin(phase)],
                       dim=-1) / norm[:, None, None, None]
    return cube.reshape(-1)


def min_conv_size_half(support: np.ndarray, oversample: int) -> int:
    """Smallest quadrant side the reference indexes without reading past a
    kernel row: oversample * S_max + ceil(oversample / 2) + 1."""
    return int(oversample * int(support.max()) + (oversample + 1) // 2 + 1)


# --------------------------------------------------------------------------
# Named configurations
# --------------------------------------------------------------------------

def _finish(name, uu, vv, ww, vis, support, oversample, csh, cell, w_scale,
            grid_size, gen, device, **meta):
    weight = torch.ones_like(uu)
    cube = analytic_kernel_cube(support, oversample, csh, device=device)
    return Workload(name=name, uu=uu, vv=vv, ww=ww, vis=vis, weight=weight,
                    support=support, oversample=oversample,
                    conv_size_half=csh, conv_func=cube, cell_size_rad=cell,
                    w_scale=w_scale, grid_size=grid_size, meta=meta)


def plain_small(seed: int = 0, device="cpu", num_stations=64, num_times=120,
                grid_size=1024, num_w_planes=16) -> Workload:
    """Plain W-projection, small: 64 stations uniform in a 1 km disk (2016
    baselines), 120 samples 10 s apart, 100 MHz, dec -30 deg (241,920
    visibilities); 10 point sources within 1 deg, noise sigma 0.1; grid
    1024^2 with cell 4 deg / 1024; 16 w-planes with
    w_scale = 15^2 / max|w|; support 4 -> 16; oversample 4."""
    gen = torch.Generator().manual_seed(seed)
    enu = stations_uniform_disk(num_stations, 1000.0, gen)
    lat = dec = math.radians(-30.0)
    uu, vv, ww = earth_rotation_uvw(baselines_xyz(enu, lat), num_times, 10.0,
                                    100e6, dec, device)
    vis = point_source_vis(uu, vv, ww, 10, math.radians(1.0), 0.1, gen)
    support = support_ramp(num_w_planes, 4, 16)
    w_scale = float((num_w_planes - 1) ** 2 / ww.abs().max().item())
    cell = math.radians(4.0) / 1024
    csh = 69
    return _finish("plain_small", uu, vv, ww, vis, support, 4, csh, cell,
                   w_scale, grid_size, gen, device, seed=seed)


def plain_large(seed: int = 1, device="cpu", num_stations=512, num_times=300,
                grid_size=8192, num_w_planes=256, oversample=4) -> Workload:
    """Plain W-projection, large single job: 512 stations log-radial out to
    30 km (130,816 baselines), 300 samples 10 s apart, 150 MHz, dec -30 deg
    (39,244,800 visibilities); sky as plain_small; grid 8192^2; 256 w-planes,
    support 4 -> 36, oversample 4, conv_size_half = 37 * 4 + 1 = 149.  The
    cell is chosen so the longest baseline plus the largest support lands
    inside the grid (no visibility is skipped)."""
    gen = torch.Generator().manual_seed(seed)
    enu = stations_log_radial(num_stations, 20.0, 30000.0, gen)
    lat = dec = math.radians(-30.0)
    uu, vv, ww = earth_rotation_uvw(baselines_xyz(enu, lat), num_times, 10.0,
                                    150e6, dec, device)
    vis = point_source_vis(uu, vv, ww, 10, math.radians(1.0), 0.1, gen)
    support = support_ramp(num_w_planes, 4, 36)
    w_scale = float((num_w_planes - 1) ** 2 / ww.abs().max().item())
    uv_max = float(torch.maximum(uu.abs().max(), vv.abs().max()).item())
    cell = (grid_size // 2 - int(support.max()) - 2) / (grid_size * uv_max)
    csh = 37 * oversample + 1
    return _finish("plain_large", uu, vv, ww, vis, support, oversample, csh,
                   cell, w_scale, grid_size, gen, device, seed=seed)


def precision_sweep(seed: int = 3, device="cpu", num_stations=512,
                    num_times=3000, grid_size=4096, num_w_planes=128,
                    oversample=8, freq_hz=150e6) -> Workload:
    """Precision sweep, long integration: 512 stations uniform in a 5 km
    disk (130,816 baselines, short ones dominating), 3000 samples 10 s apart
    at 150 MHz, dec -30 deg (392,448,000 visibilities, concentrated near the
    uv origin); sky as plain_small; grid 4096^2; 128 w-planes, support
    4 -> 32, oversample 8.  The cell is chosen so the longest baseline plus
    the largest support lands inside the grid."""
    gen = torch.Generator().manual_seed(seed)
    enu = stations_uniform_disk(num_stations, 5000.0, gen)
    lat = dec = math.radians(-30.0)
    uu, vv, ww = earth_rotation_uvw(baselines_xyz(enu, lat), num_times, 10.0,
                                    freq_hz, dec, device)
    vis = point_source_vis(uu, vv, ww, 10, math.radians(1.0), 0.1, gen)
    support = support_ramp(num_w_planes, 4, 32)
    w_scale = float((num_w_planes - 1) ** 2 / ww.abs().max().item())
    uv_max = float(torch.maximum(uu.abs().max(), vv.abs().max()).item())
    cell = (grid_size // 2 - int(support.max()) - 2) / (grid_size * uv_max)
    csh = min_conv_size_half(support, oversample) + 1
    return _finish("precision_sweep", uu, vv, ww, vis, support, oversample,
                   csh, cell, w_scale, grid_size, gen, device, seed=seed)


def batch_channels(seed: int = 2, device="cpu", num_channels=128,
                   num_stations=256, num_times=60, grid_size=2048,
                   num_w_planes=64, f_lo=50e6, f_hi=350e6, max_flag=0.7,
                   s_lo=3, s_hi=24, oversample=4) -> list:
    """Batching workload: num_channels channels spanning f_lo..f_hi, each
    gridded into its own grid with its own kernel cube.  Array: 256 stations
    uniform in a disk 10 km across (5 km radius), 60 samples 10 s apart, dec
    -30 deg (32,640 baselines, 1,958,400 visibilities per channel before
    flagging).  Seeded random flagging removes a U(0, max_flag) fraction of
    each channel.  Per channel: num_w_planes planes with support ramping from
    s_lo to s_lo + (s_hi - s_lo) * f / f_hi (scaled by frequency), w_scale =
    (P-1)^2 / max|w|, oversample 4.  One cell size for all channels, chosen
    so the highest channel's longest baseline plus its support fits.
    Returns a list of Workloads (FP64; convert with .to)."""
    gen = torch.Generator().manual_seed(seed)
    enu = stations_uniform_disk(num_stations, 5000.0, gen)
    lat = dec = math.radians(-30.0)
    bxyz = baselines_xyz(enu, lat)
    # uvw in metres (scale 1 Hz -> multiply by f / c per channel)
    um, vm, wm = earth_rotation_uvw(bxyz, num_times, 10.0, C_LIGHT, dec,
                                    device)
    freqs = torch.linspace(f_lo, f_hi, num_channels, dtype=torch.float64)
    uv_max_hi = float(torch.maximum(um.abs().max(), vm.abs().max())) * \
        f_hi / C_LIGHT
    cell = (grid_size // 2 - s_hi - 2) / (grid_size * uv_max_hi)
    out = []
    n_all = um.numel()
    for ch in range(num_channels):
        f = float(freqs[ch])
        scale = f / C_LIGHT
        keep_frac = 1.0 - max_flag * float(torch.rand(1, generator=gen))
        flags = torch.rand(n_all, generator=gen) < keep_frac
        idx = torch.nonzero(flags).squeeze(1).to(device)
        uu, vv, ww = um[idx] * scale, vm[idx] * scale, wm[idx] * scale
        vis = point_source_vis(uu, vv, ww, 10, math.radians(1.0), 0.1, gen)
        s_max = int(round(s_lo + (s_hi - s_lo) * f / f_hi))
        support = support_ramp(num_w_planes, s_lo, s_max)
        w_scale = float((num_w_planes - 1) ** 2 / ww.abs().max().item())
        csh = min_conv_size_half(support, oversample) + 1
        out.append(_finish(f"channel_{ch}", uu, vv, ww, vis, support,
                           oversample, csh, cell, w_scale, grid_size, gen,
                           device, seed=seed, channel=ch, freq_hz=f,
                           kept=keep_frac))
    return out


def serving_stream(num_jobs: int = 2000, seed: int = 4, device="cpu",
                   n_lo: float = 1e4, n_hi: float = 5e7,
                   grid_sizes=(512, 1024, 2048, 4096, 8192),
                   p_lo: int = 8, p_hi: int = 256, s_lo: int = 3,
                   s_hi: int = 32, shared_frac: float = 0.2,
                   num_shared: int = 8, num_stations: int = 512,
                   oversample: int = 4):
    """Serving workload: num_jobs gridding jobs whose visibility counts are
    log-uniform in [n_lo, n_hi], grid sizes drawn from grid_sizes, 8-256
    w-planes and a largest support of 3-32 (support ramps from 3); about
    shared_frac of the jobs use one of num_shared shared kernel-cube specs,
    the rest their own.  Every job is a contiguous slice of one base
    observation (plain_large's array: 512 stations log-radial to 30 km,
    150 MHz, 10 s samples, enough samples for n_hi visibilities), with the
    cell and w_scale chosen for that slice so nothing is skipped.
    Returns (base, jobs): base holds FP32 device tensors uu, vv, ww, vis,
    weight; each job is a dict with start, n, grid_size, cell_size_rad,
    w_scale, cube_key; cube specs are in cubes[cube_key] = (support,
    conv_size_half)."""
    rng = np.random.default_rng(seed)
    gen = torch.Generator().manual_seed(seed)
    enu = stations_log_radial(num_stations, 20.0, 30000.0, gen)
    nb = num_stations * (num_stations - 1) // 2
    num_times = int(math.ceil(n_hi / nb))
    lat = dec = math.radians(-30.0)
    uu, vv, ww = earth_rotation_uvw(baselines_xyz(enu, lat), num_times, 10.0,
                                    150e6, dec, device)
    vis = point_source_vis(uu, vv, ww, 10, math.radians(1.0), 0.1, gen)
    base = dict(uu=uu.float(), vv=vv.float(), ww=ww.float(), vis=vis.float(),
                weight=torch.ones_like(uu, dtype=torch.float32))
    total = uu.numel()

    def spec():
        p = int(rng.integers(p_lo, p_hi + 1))
        s = int(rng.integers(s_lo, s_hi + 1))
        sup = support_ramp(p, s_lo, s)
        return sup, min_conv_size_half(sup, oversample) + 1

    cubes = {}
    for k in range(num_shared):
        cubes[("shared", k)] = spec()
    jobs = []
    absu = torch.maximum(uu.abs(), vv.abs())
    absw = ww.abs()
    for j in range(num_jobs):
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        n = min(n, total)
        start = int(rng.integers(0, total - n + 1))
        g = int(rng.choice(grid_sizes))
        if rng.uniform() < shared_frac:
            key = ("shared", int(rng.integers(0, num_shared)))
        else:
            key = ("job", j)
            cubes[key] = spec()
        sup, csh = cubes[key]
        uv_max = float(absu[start:start + n].max())
        w_max = float(absw[start:start + n].max())
        cell = (g // 2 - int(sup.max()) - 2) / (g * uv_max)
        w_scale = (len(sup) - 1) ** 2 / w_max if w_max > 0 else 1.0
        jobs.append(dict(start=start, n=n, grid_size=g,
                         cell_size_rad=float(np.float32(cell)),
                         w_scale=float(np.float32(w_scale)), cube_key=key))
    return base, jobs, cubes


def scaled(workload_fn, **overrides):
    """A smaller variant of a named configuration (same generator, fewer
    stations/times/planes or a smaller grid) for quick parity runs."""
    return workload_fn(**overrides)
