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
    cube = torch.empty(num_planes, conv_size_half, conv_size_half, 2,
                       dtype=torch.float64, device=device)
    for p in range(num_planes):
        s = int(support[p])
        sigma = s / taper_div
        taper = torch.exp(-r2 / (2 * sigma * sigma))
        taps = torch.arange(-s, s + 1, device=device).abs() * oversample
        norm = taper[taps][:, taps].sum()
        phase = 2 * math.pi * chirp * p * r2
        cube[p, :, :, 0] = taper * torch.cos(phase) / norm
        cube[p, :, :, 1] = taper * torch.sin(phase) / norm
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


def scaled(workload_fn, **overrides):
    """A smaller variant of a named configuration (same generator, fewer
    stations/times/planes or a smaller grid) for quick parity runs."""
    return workload_fn(**overrides)
