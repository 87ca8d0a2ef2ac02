"""Host-side mirror of the reference's cloud subsystem API.

Same names, argument meaning and error behaviour as `CloudsSubsystem` /
`CloudsFactory` (crates/ps-clouds/src/lib.rs:95-1290) behind the
`RenderSubsystem` trait (crates/ps-core/src/subsystem.rs:66-118), driving the
CUDA march through the C ABI.  Device buffers are torch tensors (plumbing
only); every kernel launch happens inside libpsclouds.so.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field

import numpy as np

from . import capi
from .capi import call, ptr

NAME = "clouds"
PASS_MARCH, PASS_TAA, PASS_COMPOSITE = 0, 1, 2
MAX_CLOUD_LAYERS = 8
MAX_CLOUD_VIEWS = 2


class PassStage(enum.IntEnum):
    """crates/ps-core/src/subsystem.rs:16-31"""
    Compute = 0
    SkyBackdrop = 1
    Opaque = 2
    Translucent = 3
    PostProcess = 4
    ToneMap = 5
    Overlay = 6


@dataclass(frozen=True)
class PassDescriptor:
    name: str
    stage: PassStage
    id: int


@dataclass
class CloudsTuning:
    """`[render.clouds]` (crates/ps-core/src/config.rs:352-500) with its defaults."""
    cloud_steps: int = 192
    light_steps: int = 6
    multi_scatter_octaves: int = 4
    detail_strength: float = 0.35
    powder_strength: float = 1.0
    freeze_time: bool = False
    temporal_jitter: bool = False
    droplet_diameter_bias: float = 1.0
    wind_drift_strength: float = 1.0
    wind_skew_strength: float = 0.5
    diurnal_strength: float = 1.0
    half_res_render: bool = False
    temporal_taa: bool = False
    cone_light_sampling: bool = False
    forward_bias: float = 0.0


@dataclass
class WeatherInputs:
    """The parts of `WeatherState` the march reads (crates/ps-core/src/weather.rs:228-263)."""
    cloud_layers: list            # CloudLayerGpu entries
    weather_map: np.ndarray
    weather_w: int
    weather_h: int
    weather_format: int
    wind: np.ndarray
    type_grid: np.ndarray | None = None
    revision: int = 0


@dataclass
class PrepareContext:
    frame: capi.FrameUniformsGpu
    world: capi.WorldUniformsGpu
    weather: WeatherInputs


@dataclass
class RenderContext:
    color: object                 # torch (H, W, 4) float32 on the device: the HDR target
    depth: object = None          # torch (H, W) float32 reverse-Z, or None (sky)
    stream: object = None         # torch.cuda.Stream or None (current stream)
    extra: dict = field(default_factory=dict)


class CloudsSubsystem:
    """`CloudsSubsystem` (crates/ps-clouds/src/lib.rs:95)."""

    def __init__(self, tuning: CloudsTuning | None = None, device: int = 0,
                 options: capi.MarchOptions | None = None, bake_noise: bool = True):
        self._ctx = C.c_void_p()
        call("psc_create", device, C.byref(self._ctx))
        self.device = device
        self._tuning = tuning or CloudsTuning()
        self._params = capi.CloudParamsGpu()
        call("psc_params_default", C.byref(self._params))
        self._apply_tuning(self._tuning)
        self._layers_revision = None
        self._luts_ready = False
        self._cloud_rt = None
        self.active_view = 0
        self.options = options or self._default_options()
        self.options.half_res, self.options.taa = self._rt_flags(self._tuning)
        call("psc_set_options", self._ctx, C.byref(self.options))
        if bake_noise:
            call("psc_bake_noise", self._ctx)   # CloudNoise::bake (noise.rs:71)
        self._push_params()

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if self._ctx:
            capi.lib().psc_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _default_options():
        o = capi.MarchOptions()
        call("psc_options_default", C.byref(o))
        return o

    # -- RenderSubsystem ----------------------------------------------------
    def name(self) -> str:
        return NAME

    def register_passes(self) -> list[PassDescriptor]:  # lib.rs:1150-1168
        return [PassDescriptor("clouds::march", PassStage.Translucent, PASS_MARCH),
                PassDescriptor("clouds::taa", PassStage.Translucent, PASS_TAA),
                PassDescriptor("clouds::composite", PassStage.Translucent, PASS_COMPOSITE)]

    def prepare(self, ctx: PrepareContext) -> None:  # lib.rs:1105-1148
        if self._layers_revision != ctx.weather.revision:
            layers = list(ctx.weather.cloud_layers)[:MAX_CLOUD_LAYERS]
            if not layers:  # demonstration layer when synthesis supplied none (lib.rs:604-623)
                layers = [capi.CloudLayerGpu(1500.0, 3500.0, 0.4, 1.0, 0, 0.0, 0.0, 0.0, 20.0)]
            arr = (capi.CloudLayerGpu * len(layers))(*layers)
            call("psc_set_layers", self._ctx, arr, len(layers))
            w = ctx.weather
            call("psc_upload_weather", self._ctx, ptr(np.ascontiguousarray(w.weather_map)),
                 w.weather_w, w.weather_h, w.weather_format)
            if w.type_grid is not None:
                side = int(round(np.sqrt(w.type_grid.size)))
                call("psc_upload_type_grid", self._ctx, ptr(np.ascontiguousarray(w.type_grid)),
                     side, side)
            else:
                call("psc_upload_type_grid", self._ctx, None, 0, 0)
            wind = np.ascontiguousarray(w.wind, np.uint16)
            call("psc_upload_wind", self._ctx, ptr(wind), wind.size)
            self._layers_revision = w.revision
        call("psc_set_frame", self._ctx, C.byref(ctx.frame), C.byref(ctx.world))
        self._push_params()

    def dispatch_pass(self, pass_id: int, ctx: RenderContext) -> None:  # lib.rs:1170-1182
        if pass_id == PASS_MARCH:
            self._dispatch_march(ctx)
        elif pass_id == PASS_TAA:
            # With TAA active the march call already resolved the cloud RT
            # against the active view's history (psc_render's TAA form), so
            # this pass has nothing left to do (lib.rs:1000-1050).
            return
        elif pass_id == PASS_COMPOSITE:
            self._dispatch_composite(ctx)
        else:
            raise ValueError(f"clouds: unknown pass id {pass_id}")

    def reconfigure(self, tuning: CloudsTuning) -> None:  # lib.rs:1184-1224
        self._tuning = tuning
        self._apply_tuning(tuning)
        self._push_params()
        half, taa = self._rt_flags(tuning)
        if (self.options.half_res, self.options.taa) != (half, taa):
            o = capi.MarchOptions.from_buffer_copy(self.options)
            o.half_res, o.taa = half, taa
            self.set_options(o)

    # -- CloudsSubsystem API -----------------------------------------------
    def noise(self, kind: int) -> np.ndarray:
        out = np.zeros(capi.NOISE_BYTES[kind], np.uint8)
        call("psc_download_noise", self._ctx, kind, ptr(out), out.size)
        return out

    @property
    def params(self) -> capi.CloudParamsGpu:
        p = capi.CloudParamsGpu()
        call("psc_get_params", self._ctx, C.byref(p))
        return p

    def set_atmosphere_luts(self, luts: dict | None = None, stream=None) -> None:
        """Upload LUTs (dict of RGBA16F arrays) or bake them on the device (None)."""
        if luts is None:
            call("psc_bake_luts", self._ctx, _stream_handle(stream))
        else:
            for kind, key in ((capi.LUT_TRANSMITTANCE, "transmittance"),
                              (capi.LUT_MULTISCATTER, "multiscatter"),
                              (capi.LUT_SKYVIEW, "skyview"), (capi.LUT_AERIAL, "aerial")):
                a = np.ascontiguousarray(luts[key], np.uint16)
                call("psc_upload_lut", self._ctx, kind, ptr(a), a.size)
        self._luts_ready = True

    def set_march_steps(self, cloud: int, light: int) -> None:  # lib.rs:709-712
        call("psc_set_march_steps", self._ctx, cloud, light)
        self._params.cloud_steps = min(max(cloud, 8), 256)
        self._params.light_steps = min(max(light, 1), 16)

    def set_active_view(self, view: int) -> None:  # lib.rs:722
        self.active_view = min(int(view), MAX_CLOUD_VIEWS - 1)
        call("psc_set_active_view", self._ctx, self.active_view)

    def invalidate_taa_history(self) -> None:  # lib.rs:729
        call("psc_invalidate_taa_history", self._ctx)

    def set_options(self, options: capi.MarchOptions) -> None:
        call("psc_set_options", self._ctx, C.byref(options))
        self.options = options

    def set_params(self, params: capi.CloudParamsGpu) -> None:
        self._params = params
        self._push_params()

    def launch_count(self) -> int:
        n = C.c_uint64()
        call("psc_launch_count", self._ctx, C.byref(n))
        return n.value

    @property
    def handle(self) -> C.c_void_p:
        return self._ctx

    # -- internals ----------------------------------------------------------
    def _apply_tuning(self, c: CloudsTuning) -> None:  # lib.rs:569-600
        p = self._params
        p.cloud_steps, p.light_steps = c.cloud_steps, c.light_steps
        p.multi_scatter_octaves = c.multi_scatter_octaves
        p.detail_strength, p.powder_strength = c.detail_strength, c.powder_strength
        p.droplet_diameter_bias = c.droplet_diameter_bias
        p.cone_light_sampling = int(c.cone_light_sampling)
        p.forward_bias = c.forward_bias
        p.temporal_jitter = int(c.temporal_jitter and not c.freeze_time)
        p.wind_drift_strength = 0.0 if c.freeze_time else c.wind_drift_strength
        p.diurnal_strength = c.diurnal_strength
        p.wind_skew_strength = c.wind_skew_strength

    def _push_params(self) -> None:
        call("psc_set_params", self._ctx, C.byref(self._params))

    @staticmethod
    def _rt_flags(t: CloudsTuning) -> tuple[int, int]:
        """(half_res, taa) options: TAA is active when enabled and time is not
        frozen (lib.rs:776)."""
        return int(t.half_res_render), int(t.temporal_taa and not t.freeze_time)

    def _dispatch_march(self, ctx: RenderContext) -> None:
        """March into the cloud RT (half size with half_res_render, lib.rs:
        746-758); with TAA the same call resolves it against the active
        view's history."""
        import torch
        h, w = int(ctx.color.shape[0]), int(ctx.color.shape[1])
        rw, rh = C.c_uint32(), C.c_uint32()
        call("psc_cloud_rt_size", w, h, self.options.half_res, C.byref(rw), C.byref(rh))
        rw, rh = rw.value, rh.value
        if self._cloud_rt is None or self._cloud_rt[0].shape[:2] != (rh, rw):
            dev = ctx.color.device
            self._cloud_rt = (torch.zeros((rh, rw, 4), dtype=torch.float32, device=dev),
                              torch.ones((rh, rw, 4), dtype=torch.float32, device=dev))
        lum, tr = self._cloud_rt
        view = capi.View(w, h, ptr(ctx.depth).value, lum.data_ptr(), tr.data_ptr(), None)
        call("psc_render", self._ctx, C.byref(view), 1, _stream_handle(ctx.stream))

    def _dispatch_composite(self, ctx: RenderContext) -> None:
        if self._cloud_rt is None:
            return
        lum, tr = self._cloud_rt
        h, w = int(ctx.color.shape[0]), int(ctx.color.shape[1])
        rh, rw = int(lum.shape[0]), int(lum.shape[1])
        if (rh, rw) != (h, w):  # half-res RT: Catmull-Rom upsample (lib.rs:1054-1097)
            call("psc_composite_halfres", ptr(lum), ptr(tr), rw, rh, ptr(ctx.color), w, h,
                 _stream_handle(ctx.stream))
        else:
            call("psc_composite", ptr(lum), ptr(tr), ptr(ctx.color), w, h, _stream_handle(ctx.stream))

    @property
    def cloud_rt(self):
        return self._cloud_rt


class CloudsFactory:
    """`CloudsFactory` (crates/ps-clouds/src/lib.rs:1228-1290)."""

    def __init__(self, atmosphere_luts: dict | None = None):
        self.atmosphere_luts = atmosphere_luts

    def name(self) -> str:
        return NAME

    def build(self, tuning: CloudsTuning | None = None, device: int = 0) -> CloudsSubsystem:
        sub = CloudsSubsystem(tuning, device)
        if self.atmosphere_luts is not None:
            sub.set_atmosphere_luts(self.atmosphere_luts)
        return sub


def _stream_handle(stream) -> C.c_void_p:
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available():
                return C.c_void_p(torch.cuda.current_stream().cuda_stream)
        except Exception:
            pass
        return C.c_void_p(None)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


def subsystem_for_scene(scene, device=0, luts=None, noise=None) -> CloudsSubsystem:
    """A subsystem prepared with a `scenes.Scene`: params, layers, frame, weather, LUTs."""
    sub = CloudsSubsystem(device=device, options=scene.options, bake_noise=noise is None)
    if noise is not None:
        for kind, key in ((capi.NOISE_BASE, "base"), (capi.NOISE_DETAIL, "detail"),
                          (capi.NOISE_CURL, "curl"), (capi.NOISE_BLUE, "blue")):
            a = np.ascontiguousarray(noise[key], np.uint8)
            call("psc_upload_noise", sub.handle, kind, ptr(a), a.size)
    layers = [scene.layers[i] for i in range(scene.n_layers)]
    weather = WeatherInputs(layers, scene.weather, scene.weather_w, scene.weather_h,
                            scene.weather_format, scene.wind, scene.type_grid, revision=1)
    sub.set_params(scene.params)
    sub.prepare(PrepareContext(scene.frame, scene.world, weather))
    sub.set_atmosphere_luts(luts)
    return sub
