"""ORACLE — test infrastructure, not product code.

ctypes wrapper around oracle/liboracle.so, the CPU restatement of the
reference's cloud-march path.  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg may import this module; it is the checker,
never the thing measured or shipped.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

from pedalsky_b200 import capi

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

FP32, FP64 = 32, 64
FILTER_EXACT, FILTER_Q8 = 0, 1
COUNTERS = ("weather", "type", "base", "curl", "detail", "light", "trans", "sky", "wind", "ap",
            "blue", "depth", "steps", "dense", "pixels")


class OracleScene(C.Structure):
    _fields_ = [
        ("params", capi.CloudParamsGpu), ("layers", capi.CloudLayerGpu * 8),
        ("frame", capi.FrameUniformsGpu), ("world", capi.WorldUniformsGpu),
        ("options", capi.MarchOptions),
        ("noise_base", C.c_void_p), ("noise_detail", C.c_void_p), ("noise_curl", C.c_void_p),
        ("blue_noise", C.c_void_p), ("weather", C.c_void_p), ("weather_w", C.c_uint32),
        ("weather_h", C.c_uint32), ("weather_format", C.c_int), ("type_grid", C.c_void_p),
        ("type_w", C.c_uint32), ("type_h", C.c_uint32), ("wind", C.c_void_p),
        ("lut_transmittance", C.c_void_p), ("lut_skyview", C.c_void_p),
        ("lut_aerial", C.c_void_p), ("depth", C.c_void_p),
    ]


_LIB = None


def build() -> Path:
    res = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + res.stdout + res.stderr)
    return LIB_PATH


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        vp, u32, f32 = C.c_void_p, C.c_uint32, C.c_float
        for name, args, res in [
            ("oracle_bake_noise_base", [vp], C.c_int),
            ("oracle_bake_noise_detail", [vp], C.c_int),
            ("oracle_bake_noise_curl", [vp], C.c_int),
            ("oracle_blue_noise", [vp], C.c_int),
            ("oracle_params_default", [vp], C.c_int),
            ("oracle_world_default", [vp], C.c_int),
            ("oracle_remap_coverage", [f32], f32),
            ("oracle_synthesise_layers", [vp, u32, vp], C.c_int),
            ("oracle_weather_map", [u32, f32, f32, vp, u32, u32, f32, vp], C.c_int),
            ("oracle_value_noise_2d", [f32, f32], f32),
            ("oracle_wind_field", [f32, f32, vp], C.c_int),
            ("oracle_frame_from_camera", [vp, u32, u32, f32, f32, f32, f32, vp], C.c_int),
            ("oracle_f32_to_f16", [f32], C.c_uint16),
            ("oracle_f16_to_f32", [C.c_uint16], f32),
            ("oracle_bake_transmittance", [vp, vp], C.c_int),
            ("oracle_bake_multiscatter", [vp, vp, vp], C.c_int),
            ("oracle_bake_skyview", [vp, vp, vp, vp, vp], C.c_int),
            ("oracle_bake_aerial", [vp, vp, vp, vp, vp], C.c_int),
            ("oracle_render", [vp, u32, u32, C.c_int, C.c_int, C.c_int, u32, u32, vp, vp, vp], C.c_int),
            ("oracle_render_pixel", [vp, u32, u32, u32, u32, C.c_int, C.c_int, vp, vp], C.c_int),
            ("oracle_branch_margins", [vp, u32, u32, C.c_int, u32, u32, vp, vp], C.c_int),
            ("oracle_render_frozen", [vp, vp, u32, u32, C.c_int, vp, vp], C.c_longlong),
            ("oracle_composite", [vp, vp, vp, u32], C.c_int),
            ("oracle_density_sample", [vp, u32, vp, C.c_double, C.c_double, vp, vp], C.c_int),
            ("oracle_grid_render", [vp, vp, u32, u32, C.c_int, C.c_int, vp, vp], C.c_int),
            ("oracle_grid_loss", [vp, vp, u32, u32, vp, vp, vp, u32, C.c_int, vp], C.c_int),
            ("oracle_grid_adjoint", [vp, vp, u32, u32, vp, vp, u32, u32, C.c_int, vp, vp, vp],
             C.c_int),
            ("oracle_grid_fd", [vp, vp, u32, u32, vp, vp, vp, u32, C.c_double, C.c_int, vp, vp],
             C.c_int),
            ("oracle_grid_counts", [vp, vp, u32, u32, C.c_int, vp], C.c_int),
        ]:
            fn = getattr(L, name)
            fn.argtypes, fn.restype = args, res
        _LIB = L
    return _LIB


class OracleHost:
    """The scene-assembly helpers of `pedalsky_b200.scenes` (its CapiHost)
    answered by this restatement instead of the product library, so a
    process that only runs the CPU restatement (the reference arm of the
    benchmark) assembles the same scenes without mapping libpsclouds.so:

        with scenes.host_helpers(pyoracle.OracleHost()):
            s = scenes.precision_1080p()
    """

    def params_default(self, out):
        _ok(lib().oracle_params_default(C.byref(out)), "oracle_params_default")

    def world_default(self, out):
        _ok(lib().oracle_world_default(C.byref(out)), "oracle_world_default")

    def options_default(self, out):
        # PscMarchOptions' reference behaviour: approx-Mie, U8 storage, exact
        # filtering, plain schedule; the dual-lobe HG lobes at 0.8 / -0.2 / 0.5
        C.memset(C.byref(out), 0, C.sizeof(out))
        out.phase_mode = capi.PHASE_APPROX_MIE
        out.hg_g_forward, out.hg_g_backward, out.hg_blend = 0.8, -0.2, 0.5
        out.storage, out.filter, out.schedule = capi.STORAGE_U8, capi.FILTER_EXACT, capi.SCHED_PLAIN

    def synthesise_layers(self, descs, n, out):
        _ok(lib().oracle_synthesise_layers(C.cast(descs, C.c_void_p), n, C.cast(out, C.c_void_p)),
            "oracle_synthesise_layers")

    def frame_from_camera(self, cam, width, height, alt, az, ang, lux, out):
        _ok(lib().oracle_frame_from_camera(C.byref(cam), width, height, alt, az, ang, lux,
                                           C.byref(out)), "oracle_frame_from_camera")

    def weather_map(self, n_layers, grid, gw, gh, extent, out):
        _ok(lib().oracle_weather_map(n_layers, 0.0, 0.0, grid, gw, gh, extent, out),
            "oracle_weather_map")

    def wind_field(self, speed, dir_deg, out):
        _ok(lib().oracle_wind_field(speed, dir_deg, out), "oracle_wind_field")


def _p(a):
    return C.c_void_p(None) if a is None else C.c_void_p(a.ctypes.data)


def _ok(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} returned {rc}")


def bake_noise() -> dict:
    base = np.zeros(128 ** 3 * 4, np.uint8)
    detail = np.zeros(32 ** 3 * 4, np.uint8)
    curl = np.zeros(128 * 128 * 2, np.uint8)
    blue = np.zeros(64 * 64, np.uint8)
    _ok(lib().oracle_bake_noise_base(_p(base)), "base")
    _ok(lib().oracle_bake_noise_detail(_p(detail)), "detail")
    _ok(lib().oracle_bake_noise_curl(_p(curl)), "curl")
    _ok(lib().oracle_blue_noise(_p(blue)), "blue")
    return {"base": base, "detail": detail, "curl": curl, "blue": blue}


def bake_luts(frame: capi.FrameUniformsGpu, world: capi.WorldUniformsGpu) -> dict:
    L = lib()
    t = np.zeros(256 * 64 * 4, np.uint16)
    ms = np.zeros(32 * 32 * 4, np.uint16)
    sky = np.zeros(192 * 108 * 4, np.uint16)
    ap = np.zeros(32 * 32 * 64 * 4, np.uint16)
    _ok(L.oracle_bake_transmittance(C.byref(world), _p(t)), "transmittance")
    _ok(L.oracle_bake_multiscatter(C.byref(world), _p(t), _p(ms)), "multiscatter")
    _ok(L.oracle_bake_skyview(C.byref(frame), C.byref(world), _p(t), _p(ms), _p(sky)), "skyview")
    _ok(L.oracle_bake_aerial(C.byref(frame), C.byref(world), _p(t), _p(ms), _p(ap)), "aerial")
    return {"transmittance": t, "multiscatter": ms, "skyview": sky, "aerial": ap}


def make_scene(scene, noise: dict, luts: dict) -> tuple[OracleScene, list]:
    """Build an OracleScene from a pedalsky_b200.scenes.Scene; returns (struct, keepalive)."""
    keep = []

    def arr(a, dtype):
        if a is None:
            return C.c_void_p(None)
        a = np.ascontiguousarray(a, dtype)
        keep.append(a)
        return C.c_void_p(a.ctypes.data)

    s = OracleScene()
    s.params, s.frame, s.world, s.options = scene.params, scene.frame, scene.world, scene.options
    for i in range(8):
        s.layers[i] = scene.layers[i]
    s.noise_base = arr(noise["base"], np.uint8)
    s.noise_detail = arr(noise["detail"], np.uint8)
    s.noise_curl = arr(noise["curl"], np.uint8)
    s.blue_noise = arr(noise["blue"], np.uint8)
    wdt = {capi.WEATHER_RGBA16F: np.uint16, capi.WEATHER_RG8: np.uint8,
           capi.WEATHER_R32F: np.float32}[scene.weather_format]
    s.weather = arr(scene.weather, wdt)
    s.weather_w, s.weather_h, s.weather_format = scene.weather_w, scene.weather_h, scene.weather_format
    if scene.type_grid is not None:
        s.type_grid = arr(scene.type_grid, np.uint8)
        side = int(round(np.sqrt(scene.type_grid.size)))
        s.type_w = s.type_h = side
    s.wind = arr(scene.wind, np.uint16)
    s.lut_transmittance = arr(luts["transmittance"], np.uint16)
    s.lut_skyview = arr(luts["skyview"], np.uint16)
    s.lut_aerial = arr(luts["aerial"], np.uint16)
    s.depth = arr(scene.depth, np.float32)
    return s, keep


def render(scene, noise, luts, precision=FP64, filt=FILTER_EXACT, threads=0, rows=None,
           counters=False):
    """Returns (L, T[, counters]) as (h, w, 4) float32 arrays."""
    s, keep = make_scene(scene, noise, luts)
    w, h = scene.width, scene.height
    L = np.zeros((h, w, 4), np.float32)
    T = np.zeros((h, w, 4), np.float32)
    cnt = np.zeros(len(COUNTERS), np.uint64)
    r0, r1 = rows if rows else (0, 0)
    _ok(lib().oracle_render(C.byref(s), w, h, precision, filt, threads, r0, r1, _p(L), _p(T),
                            _p(cnt) if counters else C.c_void_p(None)), "oracle_render")
    del keep
    if counters:
        return L, T, dict(zip(COUNTERS, (int(c) for c in cnt)))
    return L, T


def branch_margins(scene, noise, luts, threads=0, rows=None):
    """Per-pixel relative distance of the FP64 march from its early-exit
    test (max3(T) vs 0.01) and its dense-sample test (density vs 1e-3):
    two (h, w) float64 arrays (1e30 where the test never ran)."""
    s, keep = make_scene(scene, noise, luts)
    w, h = scene.width, scene.height
    mt = np.full((h, w), 1e30)
    md = np.full((h, w), 1e30)
    r0, r1 = rows if rows else (0, 0)
    _ok(lib().oracle_branch_margins(C.byref(s), w, h, threads, r0, r1, _p(mt), _p(md)),
        "oracle_branch_margins")
    del keep
    return mt, md


def render_frozen(ref_scene, scene, noise, luts, threads=0):
    """FP64 (L, T) (float64 arrays) of `scene` with the branch outcomes (layer hits and order,
    early exits, density threshold, AP opacity test) of `ref_scene`'s march
    at each pixel, and the
    number of outcomes the replay lacked (0 when both follow one path)."""
    r, keep_r = make_scene(ref_scene, noise, luts)
    s, keep = make_scene(scene, noise, luts)
    w, h = scene.width, scene.height
    L = np.zeros((h, w, 4), np.float64)
    T = np.zeros((h, w, 4), np.float64)
    misses = lib().oracle_render_frozen(C.byref(r), C.byref(s), w, h, threads, _p(L), _p(T))
    if misses < 0:
        raise RuntimeError("oracle_render_frozen failed")
    del keep, keep_r
    return L, T, int(misses)


def density_sample(scene, noise, luts, layer, p3, alt, weather_r):
    """FP64 primary density at world point p3 (altitude alt) in `layer` with
    weather R value `weather_r`, and the layer profile ndf(h) there."""
    s, keep = make_scene(scene, noise, luts)
    p = np.ascontiguousarray(p3, np.float64)
    d, prof = C.c_double(), C.c_double()
    _ok(lib().oracle_density_sample(C.byref(s), layer, _p(p), float(alt), float(weather_r),
                                    C.byref(d), C.byref(prof)), "oracle_density_sample")
    del keep
    return d.value, prof.value


def composite(L, T, bg):
    out = np.ascontiguousarray(bg, np.float32).copy()
    _ok(lib().oracle_composite(_p(np.ascontiguousarray(L, np.float32)),
                               _p(np.ascontiguousarray(T, np.float32)), _p(out),
                               out.size // 4), "composite")
    return out


# ---- voxel-grid form (oracle_grid.cpp) ----

def grid_struct(values: np.ndarray, spec: dict) -> capi.DensityGrid:
    """PscDensityGrid over a host (ny, nz, nx) float32 array; `spec` holds
    min_x_m, min_z_m, size_x_m, size_z_m, density_scale, exit_transmittance,
    checkpoint_every."""
    ny, nz, nx = values.shape
    return capi.DensityGrid(values.ctypes.data, nx, ny, nz, spec.get("checkpoint_every", 16),
                            spec["min_x_m"], spec["min_z_m"], spec["size_x_m"], spec["size_z_m"],
                            spec["density_scale"], spec["exit_transmittance"])


def _grid_args(scene, noise, luts, values, spec):
    s, keep = make_scene(scene, noise, luts)
    v = np.ascontiguousarray(values, np.float32)
    keep.append(v)
    g = grid_struct(v, spec)
    return s, g, keep


def grid_render(scene, noise, luts, values, spec, precision=FP64, threads=0):
    s, g, keep = _grid_args(scene, noise, luts, values, spec)
    w, h = scene.width, scene.height
    L = np.zeros((h, w, 4), np.float32)
    T = np.zeros((h, w, 4), np.float32)
    _ok(lib().oracle_grid_render(C.byref(s), C.byref(g), w, h, precision, threads, _p(L), _p(T)),
        "oracle_grid_render")
    del keep
    return L, T


def grid_loss(scene, noise, luts, values, spec, bg, target, pixels=None, threads=0) -> float:
    s, g, keep = _grid_args(scene, noise, luts, values, spec)
    bg = np.ascontiguousarray(bg, np.float32)
    target = np.ascontiguousarray(target, np.float32)
    px = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
    out = C.c_double()
    _ok(lib().oracle_grid_loss(C.byref(s), C.byref(g), scene.width, scene.height, _p(bg),
                               _p(target), _p(px), 0 if px is None else px.size, threads,
                               C.byref(out)), "oracle_grid_loss")
    del keep
    return out.value


def grid_adjoint(scene, noise, luts, values, spec, bg, target, threads=0, rows=None):
    """FP64 reverse-mode gradient: (grad (ny, nz, nx) float64, d/d density_scale, loss),
    of rows [r0, r1) if `rows` is given."""
    s, g, keep = _grid_args(scene, noise, luts, values, spec)
    bg = np.ascontiguousarray(bg, np.float32)
    target = np.ascontiguousarray(target, np.float32)
    grad = np.zeros(values.shape, np.float64)
    gs, loss = C.c_double(), C.c_double()
    r0, r1 = rows if rows else (0, 0)
    _ok(lib().oracle_grid_adjoint(C.byref(s), C.byref(g), scene.width, scene.height, _p(bg),
                                  _p(target), r0, r1, threads, _p(grad), C.byref(gs),
                                  C.byref(loss)),
        "oracle_grid_adjoint")
    del keep
    return grad, gs.value, loss.value


def grid_fd(scene, noise, luts, values, spec, bg, target, voxels, eps=1e-3, threads=0):
    """Central differences of the FP64 loss at flat voxel indices: (fd, pixels touched)."""
    s, g, keep = _grid_args(scene, noise, luts, values, spec)
    bg = np.ascontiguousarray(bg, np.float32)
    target = np.ascontiguousarray(target, np.float32)
    vox = np.ascontiguousarray(voxels, np.uint64)
    out = np.zeros(vox.size, np.float64)
    npx = np.zeros(vox.size, np.uint32)
    _ok(lib().oracle_grid_fd(C.byref(s), C.byref(g), scene.width, scene.height, _p(bg), _p(target),
                             _p(vox), vox.size, eps, threads, _p(out), _p(npx)), "oracle_grid_fd")
    del keep
    return out, npx


def grid_fd_richardson(scene, noise, luts, values, spec, bg, target, voxels, eps, threads=0):
    """Central differences at eps and eps/2 combined as (4 D(eps/2) - D(eps)) / 3,
    which cancels the eps^2 truncation term: (extrapolated, D(eps), pixels touched)."""
    d1, npx = grid_fd(scene, noise, luts, values, spec, bg, target, voxels, eps, threads)
    d2, _ = grid_fd(scene, noise, luts, values, spec, bg, target, voxels, eps / 2, threads)
    return (4.0 * d2 - d1) / 3.0, d1, npx


def grid_counts(scene, noise, luts, values, spec, threads=0) -> dict:
    """Executed work of the grid forward march (see oracle_grid_counts)."""
    s, g, keep = _grid_args(scene, noise, luts, values, spec)
    out = np.zeros(5, np.uint64)
    _ok(lib().oracle_grid_counts(C.byref(s), C.byref(g), scene.width, scene.height, threads,
                                 _p(out)), "oracle_grid_counts")
    del keep
    return dict(zip(("pixels", "hit_pixels", "steps", "primary_texels", "light_texels"),
                    (int(x) for x in out)))
