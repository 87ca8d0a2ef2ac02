"""ctypes bindings for the C ABI in include/psclouds.h.

This is the same binding a Python caller of the reference-facing boundary
would write: plain structs and pointers, no torch types.  `lib()` loads the
in-tree `libpsclouds.so`; a missing library is an error, never a fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libpsclouds.so"

PSC_OK = 0
PSC_ERR = {
    -1: "INVALID_ARGUMENT", -2: "NOT_FINITE", -3: "LAYERS", -4: "MISSING_INPUT",
    -5: "CUDA", -6: "OUT_OF_MEMORY", -7: "TIMEOUT", -8: "UNSUPPORTED", -9: "DEVICE_CHECK",
}
PHASE_APPROX_MIE, PHASE_DUAL_LOBE_HG = 0, 1
STORAGE_U8, STORAGE_F32, STORAGE_F16, STORAGE_BF16, STORAGE_FP8 = range(5)
STORAGE_NAMES = {"u8": STORAGE_U8, "f32": STORAGE_F32, "f16": STORAGE_F16,
                 "bf16": STORAGE_BF16, "fp8": STORAGE_FP8}
FILTER_EXACT, FILTER_TEXTURE, FILTER_HYBRID = 0, 1, 2
FILTER_NAMES = {"exact": FILTER_EXACT, "texture": FILTER_TEXTURE, "hybrid": FILTER_HYBRID}
SCHED_PLAIN, SCHED_FAST = 0, 1
NOISE_BASE, NOISE_DETAIL, NOISE_CURL, NOISE_BLUE = range(4)
LUT_TRANSMITTANCE, LUT_MULTISCATTER, LUT_SKYVIEW, LUT_AERIAL = range(4)
LUT_SHAPES = {LUT_TRANSMITTANCE: (64, 256), LUT_MULTISCATTER: (32, 32),
              LUT_SKYVIEW: (108, 192), LUT_AERIAL: (64, 32, 32)}
WEATHER_RGBA16F, WEATHER_RG8, WEATHER_R32F = range(3)
NOISE_BYTES = {NOISE_BASE: 128 ** 3 * 4, NOISE_DETAIL: 32 ** 3 * 4,
               NOISE_CURL: 128 * 128 * 2, NOISE_BLUE: 64 * 64}

f32, u32, i32 = C.c_float, C.c_uint32, C.c_int


class CloudParamsGpu(C.Structure):
    """`CloudParamsGpu`, crates/ps-clouds/src/params.rs:33-140 (112 bytes)."""
    _fields_ = [
        ("sigma_s", f32 * 3), ("_pad_after_sigma_s", f32),
        ("sigma_a", f32 * 3), ("droplet_diameter_bias", f32),
        ("cone_light_sampling", u32), ("forward_bias", f32), ("detail_strength", f32),
        ("curl_strength", f32),
        ("powder_strength", f32), ("multi_scatter_a", f32), ("multi_scatter_b", f32),
        ("multi_scatter_c", f32),
        ("ambient_strength", f32), ("base_scale_m", f32), ("detail_scale_m", f32),
        ("weather_scale_m", f32),
        ("light_steps", u32), ("cloud_steps", u32), ("multi_scatter_octaves", u32),
        ("cloud_layer_count", u32),
        ("temporal_jitter", u32), ("wind_drift_strength", f32), ("wind_skew_strength", f32),
        ("diurnal_strength", f32),
    ]


class CloudLayerGpu(C.Structure):
    """`CloudLayerGpu`, crates/ps-core/src/weather.rs:100-134 (48 bytes)."""
    _fields_ = [
        ("base_m", f32), ("top_m", f32), ("coverage", f32), ("density_scale", f32),
        ("cloud_type", u32), ("shape_bias", f32), ("detail_bias", f32), ("anvil_bias", f32),
        ("droplet_diameter_um", f32), ("_pad_after_droplets_0", f32),
        ("_pad_after_droplets_1", f32), ("_pad_after_droplets_2", f32),
    ]


Mat4 = (f32 * 4) * 4


class FrameUniformsGpu(C.Structure):
    """`FrameUniformsGpu`, crates/ps-core/src/frame_uniforms.rs:121-160 (448 bytes)."""
    _fields_ = [
        ("view", Mat4), ("proj", Mat4), ("view_proj", Mat4), ("inv_view_proj", Mat4),
        ("camera_position_world", f32 * 4), ("camera_velocity_world", f32 * 4),
        ("sun_direction", f32 * 4), ("sun_illuminance", f32 * 4),
        ("lightning_illuminance", f32 * 4), ("lightning_origin_world", f32 * 4),
        ("viewport_size", f32 * 4),
        ("time_seconds", f32), ("simulated_seconds", f32), ("frame_index", u32), ("ev100", f32),
        ("prev_view_proj", Mat4),
    ]


class WorldUniformsGpu(C.Structure):
    """`AtmosphereParams` / `WorldUniformsGpu`, crates/ps-core/src/weather.rs:23-58 (144 bytes)."""
    _fields_ = [
        ("planet_radius_m", f32), ("atmosphere_top_m", f32), ("rayleigh_scale_height_m", f32),
        ("mie_scale_height_m", f32),
        ("rayleigh_scattering", f32 * 4), ("mie_scattering", f32 * 4), ("mie_absorption", f32 * 4),
        ("mie_g", f32), ("_pad_after_mie_g", f32 * 3),
        ("ozone_absorption", f32 * 4),
        ("ozone_center_m", f32), ("ozone_thickness_m", f32), ("_pad_after_ozone", f32 * 2),
        ("ground_albedo", f32 * 4), ("haze_extinction_per_m", f32 * 4),
    ]


class MarchOptions(C.Structure):
    _fields_ = [
        ("phase_mode", u32), ("hg_g_forward", f32), ("hg_g_backward", f32), ("hg_blend", f32),
        ("storage", u32), ("filter", u32), ("schedule", u32), ("kahan", u32), ("composite", u32),
        ("debug_checks", u32), ("tile_w", u32), ("tile_h", u32), ("half_res", u32), ("taa", u32),
        ("light_batch", u32), ("_reserved", u32),
    ]


class View(C.Structure):
    _fields_ = [
        ("width", u32), ("height", u32), ("depth", C.c_void_p),
        ("out_luminance", C.c_void_p), ("out_transmittance", C.c_void_p), ("hdr", C.c_void_p),
        ("viewport_w", u32), ("viewport_h", u32), ("x_offset", u32), ("y_offset", u32),
    ]


class CloudLayerDesc(C.Structure):
    """Scene-side `CloudLayer`, crates/ps-core/src/scene.rs:410-480; negative = per-type default."""
    _fields_ = [
        ("cloud_type", u32), ("base_m", f32), ("top_m", f32), ("coverage", f32),
        ("density_scale", f32), ("shape_octave_bias", f32), ("detail_octave_bias", f32),
        ("anvil_bias", f32), ("droplet_diameter_um", f32),
    ]


class FlyCamera(C.Structure):
    """`FlyCamera`, crates/ps-core/src/camera.rs:11-40."""
    _fields_ = [
        ("position", f32 * 3), ("pitch_rad", f32), ("yaw_rad", f32), ("roll_rad", f32),
        ("fov_y_rad", f32), ("near_m", f32),
    ]


class BatchView(C.Structure):
    """`PscBatchView`: one view of a batch with its own scene and outputs."""
    _fields_ = [
        ("frame", FrameUniformsGpu), ("params", CloudParamsGpu), ("layers", CloudLayerGpu * 8),
        ("n_layers", u32), ("width", u32), ("height", u32), ("_pad0", u32),
        ("depth", C.c_void_p), ("out_luminance", C.c_void_p), ("out_transmittance", C.c_void_p),
        ("hdr", C.c_void_p),
    ]


BATCH_PERSISTENT, BATCH_PER_VIEW = 0, 1


class BatchTuning(C.Structure):
    _fields_ = [("threads", u32), ("tile_w", u32), ("use_graph", u32), ("form", u32)]


class DensityGrid(C.Structure):
    _fields_ = [("values", C.c_void_p), ("nx", u32), ("ny", u32), ("nz", u32),
                ("checkpoint_every", u32), ("min_x_m", C.c_float), ("min_z_m", C.c_float),
                ("size_x_m", C.c_float), ("size_z_m", C.c_float), ("density_scale", C.c_float),
                ("exit_transmittance", C.c_float)]


assert C.sizeof(DensityGrid) == 48


class FetchPeaks(C.Structure):
    _fields_ = [("l2_read_gbs", f32), ("l1_read_gbs", f32), ("tex_trilinear_gfetch_s", f32),
                ("_reserved", f32)]


class FetchCounts(C.Structure):
    """`PscFetchCounts`: fetches issued by the FAST march, by kind."""
    _fields_ = [(n, C.c_uint64) for n in (
        "rays", "primary_steps", "live_steps", "weather_taps", "type_loads", "detail_taps",
        "dense_samples", "light_taps", "transmittance_taps", "skyview_taps", "ap_taps",
        "depth_loads", "dense_warp_passes", "dense_warp_lanes")]

    def as_dict(self) -> dict:
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


class PscError(RuntimeError):
    def __init__(self, code: int, func: str, msg: str):
        super().__init__(f"{func}: {PSC_ERR.get(code, code)} ({code}): {msg}")
        self.code = code


P = C.POINTER
_vp = C.c_void_p
# name -> argtypes (all return int unless listed in _RESTYPES)
_PROTOS = {
    "psc_last_error": [],
    "psc_abi_version": [],
    "psc_build_id": [],
    "psc_sizeof_params": [], "psc_sizeof_layer": [], "psc_sizeof_frame": [], "psc_sizeof_world": [],
    "psc_params_default": [P(CloudParamsGpu)],
    "psc_world_default": [P(WorldUniformsGpu)],
    "psc_options_default": [P(MarchOptions)],
    "psc_synthesise_layers": [P(CloudLayerDesc), u32, P(CloudLayerGpu)],
    "psc_frame_from_camera": [P(FlyCamera), u32, u32, f32, f32, f32, f32, P(FrameUniformsGpu)],
    "psc_generate_blue_noise": [_vp],
    "psc_synthesise_weather_map": [u32, f32, f32, _vp, u32, u32, f32, _vp],
    "psc_synthesise_wind_field": [f32, f32, _vp],
    "psc_create": [i32, P(_vp)],
    "psc_destroy": [_vp],
    "psc_set_march_steps": [_vp, u32, u32],
    "psc_set_params": [_vp, P(CloudParamsGpu)],
    "psc_get_params": [_vp, P(CloudParamsGpu)],
    "psc_set_layers": [_vp, P(CloudLayerGpu), u32],
    "psc_set_frame": [_vp, P(FrameUniformsGpu), P(WorldUniformsGpu)],
    "psc_set_options": [_vp, P(MarchOptions)],
    "psc_get_options": [_vp, P(MarchOptions)],
    "psc_bake_noise": [_vp],
    "psc_upload_noise": [_vp, i32, _vp, C.c_size_t],
    "psc_download_noise": [_vp, i32, _vp, C.c_size_t],
    "psc_upload_weather": [_vp, _vp, u32, u32, i32],
    "psc_upload_type_grid": [_vp, _vp, u32, u32],
    "psc_upload_wind": [_vp, _vp, C.c_size_t],
    "psc_upload_lut": [_vp, i32, _vp, C.c_size_t],
    "psc_bake_luts": [_vp, _vp],
    "psc_download_lut": [_vp, i32, _vp, C.c_size_t],
    "psc_render": [_vp, P(View), u32, _vp],
    "psc_composite": [_vp, _vp, _vp, u32, u32, _vp],
    "psc_count_fetches": [_vp, P(View), P(FetchCounts), _vp],
    "psc_launch_count": [_vp, P(C.c_uint64)],
    "psc_set_batch_tuning": [_vp, P(BatchTuning)],
    "psc_get_batch_tuning": [_vp, P(BatchTuning)],
    "psc_render_batch": [_vp, P(BatchView), u32, _vp],
    "psc_render_batch_noalloc": [_vp, P(BatchView), u32, _vp, _vp, _vp],
    "psc_autotune_batch": [_vp, P(BatchView), u32, u32, P(BatchTuning), P(C.c_float), _vp],
    "psc_autotune_steps": [_vp, P(BatchView), u32, C.c_float, C.c_float, u32, P(C.c_float), P(C.c_float),
                           _vp],
    "psc_render_grid": [_vp, P(DensityGrid), P(View), _vp],
    "psc_adjoint": [_vp, P(DensityGrid), P(View), _vp, _vp, _vp, _vp, _vp, _vp],
    "psc_layer_gradient": [_vp, P(DensityGrid), P(View), _vp, _vp, _vp, _vp],
    "psc_layer_param_gradient": [_vp, P(View), u32, _vp, _vp, _vp, _vp, _vp],
    "psc_measure_fetch_peaks": [i32, P(FetchPeaks), _vp],
    "psc_cloud_rt_size": [u32, u32, u32, P(u32), P(u32)],
    "psc_taa_resolve": [_vp, _vp, _vp, u32, u32, _vp, _vp, _vp],
    "psc_set_active_view": [_vp, u32],
    "psc_invalidate_taa_history": [_vp],
    "psc_composite_halfres": [_vp, _vp, u32, u32, _vp, u32, u32, _vp],
}
_RESTYPES = {
    "psc_last_error": C.c_char_p, "psc_abi_version": u32, "psc_build_id": C.c_char_p, "psc_sizeof_params": C.c_size_t,
    "psc_sizeof_layer": C.c_size_t, "psc_sizeof_frame": C.c_size_t, "psc_sizeof_world": C.c_size_t,
}
EXPORTED = tuple(_PROTOS)

_LIB = None


def lib() -> C.CDLL:
    """Load libpsclouds.so (built by `python -m pedalsky_b200.build`)."""
    global _LIB
    if _LIB is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m pedalsky_b200.build` "
                "(the CUDA path has no CPU fallback)")
        _LIB = C.CDLL(str(LIB_PATH))
        for name, args in _PROTOS.items():
            fn = getattr(_LIB, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, C.c_int)
    return _LIB


def call(name: str, *args) -> None:
    """Call an int-status entry point; raise PscError on failure."""
    rc = getattr(lib(), name)(*args)
    if rc != PSC_OK:
        raise PscError(rc, name, lib().psc_last_error().decode(errors="replace"))


def ptr(a) -> C.c_void_p:
    """void* of a numpy array, a torch tensor or an int address (None -> NULL)."""
    if a is None:
        return C.c_void_p(None)
    if isinstance(a, int):
        return C.c_void_p(a)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return C.c_void_p(a.ctypes.data)
