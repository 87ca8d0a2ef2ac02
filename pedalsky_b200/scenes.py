"""Seeded synthetic scenes for the cloud-march workloads.

Every scene is assembled the way the reference's headless render assembles
one (crates/ps-app/src/test_harness.rs:335-390): `CloudParamsGpu::default()`
overridden by the `[render.clouds]` tuning defaults
(crates/ps-core/src/config.rs:469-488 via crates/ps-clouds/src/lib.rs:561-600),
layers through `synthesise_cloud_layers`, the reference weather map and wind
field, frame uniforms from a `FlyCamera`, and determinism switches as the
golden harness sets them (wind drift 0, diurnal 0, simulated_seconds 0;
crates/ps-app/tests/golden.rs:112,119).

All host arithmetic goes through the C ABI helpers of libpsclouds.so by
default; `host_helpers(h)` swaps in another implementation of the same seven
helpers (defaults, layer synthesis, camera, weather map, wind field) for the
duration of a `with` block, which is how a CPU-only caller assembles the same
scenes without mapping the library.
Workloads:
  plain_320x180   one Cumulus layer 1500-2300 m, coverage 0.5, 320x180,
                  64/6 steps, 3 octaves, dual-lobe HG 0.8/-0.2 w=0.5
  plain_literal   the same with the 512^2 RG8 weather map 0.5+0.15*noise
  precision_1080p Cumulus 1500-2300 (0.5), Altostratus 4000-5000 (0.7),
                  Cirrus 8000-9000 (0.3), 1920x1080, 128/6 steps
  stress_2160p    Cumulonimbus 600-12000 m, coverage 0.8, 2048^2 f32
                  coverage grid, 3840x2160, 256/8 steps, 15 m/s wind
  grid_512        256x256x64 Worley voxel grid over 20x20x2 km from 1500 m,
                  512x512, 96/6 steps (the differentiable form)
"""
from __future__ import annotations

import ctypes as C
import math
from contextlib import contextmanager
from dataclasses import dataclass, field

import numpy as np

from . import capi
from .capi import call

CLOUD_TYPES = ("Cumulus", "Stratus", "Stratocumulus", "Altocumulus", "Altostratus",
               "Cirrus", "Cirrostratus", "Cumulonimbus")
TOA_LUX = 127500.0          # crates/ps-core/src/world.rs:139-146
SUN_ANGULAR_RADIUS = math.radians(0.27)  # config.rs:343


@dataclass
class Scene:
    name: str
    width: int
    height: int
    params: capi.CloudParamsGpu
    layers: object                      # CloudLayerGpu * 8
    n_layers: int
    frame: capi.FrameUniformsGpu
    world: capi.WorldUniformsGpu
    options: capi.MarchOptions
    weather: np.ndarray
    weather_w: int
    weather_h: int
    weather_format: int
    wind: np.ndarray                    # 32x16x32x4 float16 bits (uint16)
    type_grid: np.ndarray | None = None
    depth: np.ndarray | None = None     # (h, w) float32 reverse-Z, 0 = sky
    background: np.ndarray | None = None  # (h, w, 4) float32 HDR backdrop
    extra: dict = field(default_factory=dict)


class CapiHost:
    """Scene-assembly host arithmetic through the library's C ABI helpers."""

    def params_default(self, out: capi.CloudParamsGpu) -> None:
        call("psc_params_default", C.byref(out))

    def world_default(self, out: capi.WorldUniformsGpu) -> None:
        call("psc_world_default", C.byref(out))

    def options_default(self, out: capi.MarchOptions) -> None:
        call("psc_options_default", C.byref(out))

    def synthesise_layers(self, descs, n: int, out) -> None:
        call("psc_synthesise_layers", descs, n, out)

    def frame_from_camera(self, cam, width, height, alt, az, ang, lux, out) -> None:
        call("psc_frame_from_camera", C.byref(cam), width, height, alt, az, ang, lux, C.byref(out))

    def weather_map(self, n_layers: int, grid, gw: int, gh: int, extent: float, out) -> None:
        call("psc_synthesise_weather_map", n_layers, 0.0, 0.0, grid, gw, gh, extent, out)

    def wind_field(self, speed: float, dir_deg: float, out) -> None:
        call("psc_synthesise_wind_field", speed, dir_deg, out)


_HOST = CapiHost()


@contextmanager
def host_helpers(helpers):
    """Assemble scenes with `helpers` (an object with CapiHost's methods)."""
    global _HOST
    prev, _HOST = _HOST, helpers
    try:
        yield helpers
    finally:
        _HOST = prev


def default_params() -> capi.CloudParamsGpu:
    """CloudParamsGpu::default() + CloudsTuning::default() as CloudsSubsystem::new applies it."""
    p = capi.CloudParamsGpu()
    _HOST.params_default(p)
    p.cloud_steps, p.light_steps, p.multi_scatter_octaves = 192, 6, 4
    p.detail_strength = 0.35       # CloudsTuning::default (config.rs:484)
    p.powder_strength = 1.0
    p.wind_drift_strength = 0.0    # golden determinism
    p.diurnal_strength = 0.0
    p.wind_skew_strength = 0.5
    return p


def world_default() -> capi.WorldUniformsGpu:
    w = capi.WorldUniformsGpu()
    _HOST.world_default(w)
    return w


def options(phase=capi.PHASE_APPROX_MIE, storage=capi.STORAGE_U8, filt=capi.FILTER_EXACT,
            schedule=capi.SCHED_PLAIN, kahan=0, composite=0) -> capi.MarchOptions:
    o = capi.MarchOptions()
    _HOST.options_default(o)
    o.phase_mode, o.storage, o.filter, o.schedule = phase, storage, filt, schedule
    o.kahan, o.composite = kahan, composite
    return o


def synth_layers(descs: list[tuple]) -> tuple[object, int]:
    """descs: (type, base, top, coverage[, density_scale]); returns (CloudLayerGpu*8, n)."""
    n = len(descs)
    arr = (capi.CloudLayerDesc * max(n, 1))()
    for i, d in enumerate(descs):
        t, base, top, cov = d[:4]
        dens = d[4] if len(d) > 4 else -1.0
        arr[i] = capi.CloudLayerDesc(t, base, top, cov, dens, 0.0, 0.0, -1.0, -1.0)
    out = (capi.CloudLayerGpu * 8)()
    _HOST.synthesise_layers(arr, n, out)
    return out, n


def frame_for(width, height, cam_pos=(0.0, 100.0, 0.0), pitch_deg=10.0, yaw_deg=0.0,
              fov_deg=90.0, sun_alt_deg=35.0, sun_az_deg=240.0, sim_seconds=0.0):
    cam = capi.FlyCamera((C.c_float * 3)(*cam_pos), math.radians(pitch_deg), math.radians(yaw_deg),
                         0.0, math.radians(fov_deg), 0.1)
    f = capi.FrameUniformsGpu()
    _HOST.frame_from_camera(cam, width, height, math.radians(sun_alt_deg), math.radians(sun_az_deg),
                            SUN_ANGULAR_RADIUS, TOA_LUX, f)
    f.simulated_seconds = sim_seconds
    return f


def reference_weather(n_layers: int, grid: np.ndarray | None = None, grid_extent=32000.0):
    out = np.zeros(128 * 128 * 4, np.uint16)
    if grid is None:
        _HOST.weather_map(n_layers, None, 0, 0, 0.0, capi.ptr(out))
    else:
        g = np.ascontiguousarray(grid, np.float32)
        _HOST.weather_map(n_layers, capi.ptr(g), g.shape[1], g.shape[0], grid_extent, capi.ptr(out))
    return out


def wind_field(speed=5.0, dir_deg=240.0):
    """Surface::default() wind (scene.rs:217-218) unless given."""
    out = np.zeros(32 * 16 * 32 * 4, np.uint16)
    _HOST.wind_field(speed, dir_deg, capi.ptr(out))
    return out


def _hash2(x, y):
    """weather_map.rs:178-183 on int32 arrays (u32 wrap)."""
    h = (x.astype(np.uint32) * np.uint32(2654435761)).astype(np.uint32)
    h ^= (y.astype(np.uint32) * np.uint32(2246822519)).astype(np.uint32)
    h ^= h >> np.uint32(16)
    h = (h * np.uint32(2654435761)).astype(np.uint32)
    h ^= h >> np.uint32(13)
    return np.clip(h.astype(np.float32) / np.float32(4294967296.0), 0, 1)


def value_noise(x, y):
    """value_noise_2d, weather_map.rs:160-176 (float32)."""
    x = np.asarray(x, np.float32)
    y = np.asarray(y, np.float32)
    xi, yi = np.floor(x), np.floor(y)
    xf, yf = x - xi, y - yi
    ix, iy = xi.astype(np.int32), yi.astype(np.int32)
    h00, h10 = _hash2(ix, iy), _hash2(ix + 1, iy)
    h01, h11 = _hash2(ix, iy + 1), _hash2(ix + 1, iy + 1)
    sx = xf * xf * (np.float32(3) - np.float32(2) * xf)
    sy = yf * yf * (np.float32(3) - np.float32(2) * yf)
    b = h00 + (h10 - h00) * sx
    t = h01 + (h11 - h01) * sx
    return (b + (t - b) * sy).astype(np.float32)


def literal_weather_rg8(size=512):
    """512^2 RG8: R = 0.5 + 0.15 * value_noise at the reference map's spatial
    frequency (0.05 per 250 m texel), G = cloud type 0."""
    yy, xx = np.mgrid[0:size, 0:size].astype(np.float32)
    s = np.float32(0.05 * 128.0 / size)
    vn = value_noise(xx * s, yy * s)
    r = np.clip(np.rint((np.float32(0.5) + np.float32(0.15) * vn) * 255.0), 0, 255).astype(np.uint8)
    rg = np.zeros((size, size, 2), np.uint8)
    rg[..., 0] = r
    return rg.reshape(-1)


def view_rays(frame: capi.FrameUniformsGpu, width: int, height: int):
    """Per-pixel world directions (float64) as compute_view_ray builds them."""
    inv = np.array(frame.inv_view_proj, np.float64)  # [col][row]
    cam = np.array(frame.camera_position_world[:3], np.float64)
    xs = (np.arange(width) + 0.5) / width * 2 - 1
    ys = 1 - (np.arange(height) + 0.5) / height * 2
    nx, ny = np.meshgrid(xs, ys)
    h = (inv[0][None, None, :] * nx[..., None] + inv[1][None, None, :] * ny[..., None]
         + inv[2][None, None, :] + inv[3][None, None, :])
    p = h[..., :3] / h[..., 3:4]
    d = p - cam
    return d / np.linalg.norm(d, axis=-1, keepdims=True)


def ground_depth(frame, world, width, height):
    """Headless ground: reverse-Z depth of the planet sphere (0 where the ray sees sky)."""
    d = view_rays(frame, width, height)
    cam = np.array(frame.camera_position_world[:3], np.float64)
    R = float(world.planet_radius_m)
    oc = cam + np.array([0.0, R, 0.0])
    b = d @ oc
    c = oc @ oc - R * R
    disc = b * b - c
    hit = disc >= 0
    t = -b - np.sqrt(np.where(hit, disc, 0))
    hit &= t > 0
    X = cam + d * t[..., None]
    vp = np.array(frame.view_proj, np.float64)
    clip = vp[0] * X[..., 0:1] + vp[1] * X[..., 1:2] + vp[2] * X[..., 2:3] + vp[3]
    with np.errstate(divide="ignore", invalid="ignore"):
        depth = np.where(hit, clip[..., 2] / clip[..., 3], 0.0)
    return depth.astype(np.float32)


def sky_background(frame, width, height):
    """Smooth HDR backdrop the composite blends over (cd/m^2 scale)."""
    d = view_rays(frame, width, height)
    up = np.clip(d[..., 1], -1, 1)
    sky = 2500.0 + 6000.0 * (1.0 - np.abs(up)) ** 2
    tint = np.array([0.72, 0.86, 1.0])
    bg = np.empty((height, width, 4), np.float32)
    bg[..., :3] = (sky[..., None] * tint).astype(np.float32)
    bg[..., :3] = np.where(up[..., None] < 0, 900.0 * np.array([0.55, 0.5, 0.45]), bg[..., :3])
    bg[..., 3] = 1.0
    return bg


def device_inputs(frame, world, width, height, device):
    """(depth, background) of `ground_depth` / `sky_background` computed with
    torch on `device` (float64 rays), for large batches."""
    import torch
    dt = torch.float64
    inv = torch.tensor(np.array(frame.inv_view_proj, np.float64), dtype=dt, device=device)
    vp = torch.tensor(np.array(frame.view_proj, np.float64), dtype=dt, device=device)
    cam = torch.tensor(np.array(frame.camera_position_world[:3], np.float64), dtype=dt, device=device)
    xs = (torch.arange(width, dtype=dt, device=device) + 0.5) / width * 2 - 1
    ys = 1 - (torch.arange(height, dtype=dt, device=device) + 0.5) / height * 2
    ny, nx = torch.meshgrid(ys, xs, indexing="ij")
    h = inv[0] * nx[..., None] + inv[1] * ny[..., None] + inv[2] + inv[3]
    d = h[..., :3] / h[..., 3:4] - cam
    d = d / torch.linalg.norm(d, dim=-1, keepdim=True)
    R = float(world.planet_radius_m)
    oc = cam + torch.tensor([0.0, R, 0.0], dtype=dt, device=device)
    b = d @ oc
    c = oc @ oc - R * R
    disc = b * b - c
    t = -b - torch.sqrt(torch.clamp(disc, min=0))
    hit = (disc >= 0) & (t > 0)
    X = cam + d * t[..., None]
    clip = vp[0] * X[..., 0:1] + vp[1] * X[..., 1:2] + vp[2] * X[..., 2:3] + vp[3]
    depth = torch.where(hit, clip[..., 2] / clip[..., 3], torch.zeros_like(t)).float()
    up = d[..., 1].clamp(-1, 1)
    sky = 2500.0 + 6000.0 * (1.0 - up.abs()) ** 2
    tint = torch.tensor([0.72, 0.86, 1.0], dtype=dt, device=device)
    ground = torch.tensor([0.55, 0.5, 0.45], dtype=dt, device=device) * 900.0
    rgb = torch.where(up[..., None] < 0, ground.expand(height, width, 3), sky[..., None] * tint)
    bg = torch.cat([rgb, torch.ones_like(rgb[..., :1])], dim=-1).float().contiguous()
    return depth.contiguous(), bg


def _finish(name, width, height, params, layers_n, frame, opts, weather, ww, wh, wfmt,
            type_grid=None, with_ground=True, wind=None, host_inputs=True):
    layers, n = layers_n
    world = world_default()
    params.cloud_layer_count = n
    depth = ground_depth(frame, world, width, height) if (with_ground and host_inputs) else None
    bg = sky_background(frame, width, height) if host_inputs else None
    return Scene(name, width, height, params, layers, n, frame, world, opts, weather, ww, wh, wfmt,
                 wind if wind is not None else wind_field(), type_grid, depth, bg)


def plain_320x180(width=320, height=180, phase=capi.PHASE_DUAL_LOBE_HG, **kw) -> Scene:
    p = default_params()
    p.cloud_steps, p.light_steps, p.multi_scatter_octaves = 64, 6, 3
    ln = synth_layers([(0, 1500.0, 2300.0, 0.5, 1.0)])
    frame = frame_for(width, height)
    return _finish("plain_320x180", width, height, p, ln, frame, options(phase=phase, **kw),
                   reference_weather(ln[1]), 128, 128, capi.WEATHER_RGBA16F)


def plain_literal(width=320, height=180, **kw) -> Scene:
    s = plain_320x180(width, height, **kw)
    s.name = "plain_literal"
    s.weather, s.weather_w, s.weather_h = literal_weather_rg8(), 512, 512
    s.weather_format = capi.WEATHER_RG8
    s.type_grid = np.zeros(512 * 512, np.uint8)
    return s


def precision_1080p(width=1920, height=1080, steps=128, **kw) -> Scene:
    p = default_params()
    p.cloud_steps, p.light_steps = steps, 6
    ln = synth_layers([(0, 1500.0, 2300.0, 0.5), (4, 4000.0, 5000.0, 0.7),
                       (5, 8000.0, 9000.0, 0.3)])
    frame = frame_for(width, height)
    return _finish("precision_1080p", width, height, p, ln, frame, options(**kw),
                   reference_weather(ln[1]), 128, 128, capi.WEATHER_RGBA16F)


def mountain_wave_grid(size=2048, seed=0, wavelength_m=8000.0, amplitude=0.3, extent=32000.0):
    """2048^2 f32 coverage grid: mountain-wave sinusoid + seeded value noise."""
    rng = np.random.default_rng(seed)
    off = rng.uniform(0, 1000, 2).astype(np.float32)
    x = (np.arange(size, dtype=np.float32) + 0.5) / size * extent - extent / 2
    X, Y = np.meshgrid(x, x)
    wave = amplitude * np.sin(2 * np.pi * X / wavelength_m)
    vn = value_noise(X / 1500.0 + off[0], Y / 1500.0 + off[1])
    return np.clip(0.55 + wave + 0.35 * (vn - 0.5), 0, 1).astype(np.float32)


def stress_2160p(width=3840, height=2160, frame_index=0, host_inputs=True, **kw) -> Scene:
    p = default_params()
    p.cloud_steps, p.light_steps = 256, 8
    p.wind_drift_strength = 1.0
    ln = synth_layers([(7, 600.0, 12000.0, 0.8)])
    frame = frame_for(width, height, sim_seconds=float(frame_index))
    grid = mountain_wave_grid()
    s = _finish("stress_2160p", width, height, p, ln, frame, options(**kw), grid.reshape(-1),
                2048, 2048, capi.WEATHER_R32F, wind=wind_field(15.0 / 1.0, 240.0),
                host_inputs=host_inputs)
    s.extra["frame_index"] = frame_index
    return s


# Altitude bands that keep randomly typed layers disjoint: low, middle, high.
_BANDS = ((600.0, 2600.0), (3000.0, 6000.0), (7000.0, 11000.0))
CUBE_FACES = ((0.0, 0.0), (90.0, 0.0), (180.0, 0.0), (270.0, 0.0), (0.0, 89.9), (0.0, -89.9))
FRAME_SIZES = ((640, 360), (1280, 720), (1920, 1080), (2560, 1440), (3840, 2160))
CUBE_SIZES = (256, 512, 768, 1024)


def batch_views(n=64, seed=0, size_scale=1.0, host_inputs=True, **kw) -> list[Scene]:
    """Seeded batch of uneven views: half cube-map faces (256^2..1024^2,
    fov 90), half 16:9 frames (640x360..3840x2160, fov 60); each with 1-3
    disjoint layers of uniformly drawn type, coverage U[0.2, 0.9], sun
    elevation U[5, 70] deg, azimuth U[0, 360), and 48..160 primary steps.
    `size_scale` shrinks every view (tests)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        if i % 2 == 0:
            side = int(CUBE_SIZES[rng.integers(len(CUBE_SIZES))])
            w = h = side
            yaw, pitch = CUBE_FACES[rng.integers(len(CUBE_FACES))]
            fov = 90.0
        else:
            w, h = FRAME_SIZES[rng.integers(len(FRAME_SIZES))]
            yaw, pitch, fov = float(rng.uniform(0, 360)), float(rng.uniform(-5, 30)), 60.0
        w, h = max(8, int(w * size_scale)), max(8, int(h * size_scale))
        nl = int(rng.integers(1, 4))
        bands = sorted(rng.choice(3, size=nl, replace=False))
        descs = []
        for b in bands:
            lo, hi = _BANDS[b]
            t = int(rng.integers(0, 8))
            thick = float(rng.uniform(400.0, 1800.0))
            base = float(rng.uniform(lo, hi - thick))
            descs.append((t, base, base + thick, float(rng.uniform(0.2, 0.9))))
        p = default_params()
        p.cloud_steps = int(rng.integers(48, 161))
        ln = synth_layers(descs)
        frame = frame_for(w, h, yaw_deg=yaw, pitch_deg=pitch, fov_deg=fov,
                          sun_alt_deg=float(rng.uniform(5, 70)), sun_az_deg=float(rng.uniform(0, 360)))
        sc = _finish(f"batch_{i}", w, h, p, ln, frame, options(schedule=capi.SCHED_FAST, **kw),
                     reference_weather(ln[1]), 128, 128, capi.WEATHER_RGBA16F,
                     host_inputs=host_inputs)
        out.append(sc)
    return out


def worley_grid(nx=256, ny=64, nz=256, extent=(20000.0, 2000.0, 20000.0), seed=0, n_points=48,
                radius_m=1100.0, flatten=2.5, vmax=0.05):
    """Seeded Worley-thresholded voxel density, shape (ny, nz, nx), values in
    [0, vmax] 1/m: vmax * clamp(1 - F1 / radius, 0, 1), F1 the distance from
    the cell centre to the nearest of `n_points` uniformly placed feature
    points, with vertical distances scaled by `flatten` (flat-based blobs)."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    ex, ey, ez = extent
    pts = rng.uniform((0.0, 0.0, 0.0), (ex, ey, ez), size=(n_points, 3))
    pts[:, 1] *= flatten
    xs = (np.arange(nx) + 0.5) * (ex / nx)
    ys = (np.arange(ny) + 0.5) * (ey / ny) * flatten
    zs = (np.arange(nz) + 0.5) * (ez / nz)
    Y, Z, X = np.meshgrid(ys, zs, xs, indexing="ij")
    f1, _ = cKDTree(pts).query(np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1))
    v = vmax * np.clip(1.0 - f1 / radius_m, 0.0, 1.0)
    return v.reshape(ny, nz, nx).astype(np.float32)


def grid_target_values(values: np.ndarray, seed=1, rel=0.05) -> np.ndarray:
    """The grid perturbed by `rel` relative Gaussian noise (the target's density)."""
    rng = np.random.default_rng(seed)
    return np.clip(values * (1.0 + rel * rng.standard_normal(values.shape)), 0.0, None).astype(np.float32)


def grid_512(width=512, height=512, seed=0, grid_shape=(256, 64, 256), steps=96, **kw) -> Scene:
    """Voxel-grid scene: (nx, ny, nz) cells over 20 x 20 km from -10 km, 1500-3500 m
    altitude (one Cumulus layer supplies droplet size and type), camera at
    100 m pitched up 55 deg with a 60 deg field of view, `steps` + 6 steps."""
    p = default_params()
    p.cloud_steps, p.light_steps = steps, 6
    ln = synth_layers([(0, 1500.0, 3500.0, 0.5)])
    frame = frame_for(width, height, pitch_deg=55.0, fov_deg=60.0)
    s = _finish("grid_512", width, height, p, ln, frame, options(**kw), reference_weather(ln[1]),
                128, 128, capi.WEATHER_RGBA16F, with_ground=False)
    nx, ny, nz = grid_shape
    s.extra["grid"] = worley_grid(nx, ny, nz, seed=seed)
    s.extra["grid_spec"] = dict(min_x_m=-10000.0, min_z_m=-10000.0, size_x_m=20000.0,
                                size_z_m=20000.0, density_scale=1.0, exit_transmittance=0.01,
                                checkpoint_every=16)
    return s


WORKLOADS = {
    "plain_320x180": plain_320x180,
    "plain_literal": plain_literal,
    "precision_1080p": precision_1080p,
    "stress_2160p": stress_2160p,
    "batch_64": batch_views,
    "grid_512": grid_512,
}
