"""C-ABI contract tests (no GPU): struct layouts, exported symbols, host-side
validation.  Layouts are pinned to the reference's own layout tests:
crates/ps-clouds/src/params.rs:220-231 (CloudParamsGpu 112 B),
crates/ps-core/src/weather.rs:537-555 (CloudLayerGpu 48 B),
crates/ps-core/src/frame_uniforms.rs:200-210 (FrameUniformsGpu 448 B) and the
per-field std140 offsets of crates/ps-app/tests/wgsl_layout.rs:100-230."""
import ctypes as C
import math
import re
from pathlib import Path

import numpy as np
import pytest

from pedalsky_b200 import capi
from pedalsky_b200.capi import PscError, call

ROOT = Path(__file__).resolve().parent.parent


def test_struct_sizes_match_reference():
    assert C.sizeof(capi.CloudParamsGpu) == 112
    assert C.sizeof(capi.CloudLayerGpu) == 48
    assert C.sizeof(capi.FrameUniformsGpu) == 448
    assert C.sizeof(capi.WorldUniformsGpu) == 144
    L = capi.lib()
    assert L.psc_sizeof_params() == 112
    assert L.psc_sizeof_layer() == 48
    assert L.psc_sizeof_frame() == 448
    assert L.psc_sizeof_world() == 144


@pytest.mark.parametrize("field,offset", [
    ("sigma_s", 0), ("sigma_a", 16), ("droplet_diameter_bias", 28), ("cone_light_sampling", 32),
    ("forward_bias", 36), ("detail_strength", 40), ("curl_strength", 44), ("powder_strength", 48),
    ("multi_scatter_a", 52), ("multi_scatter_b", 56), ("multi_scatter_c", 60),
    ("ambient_strength", 64), ("base_scale_m", 68), ("detail_scale_m", 72),
    ("weather_scale_m", 76), ("light_steps", 80), ("cloud_steps", 84),
    ("multi_scatter_octaves", 88), ("cloud_layer_count", 92), ("temporal_jitter", 96),
    ("wind_drift_strength", 100), ("wind_skew_strength", 104), ("diurnal_strength", 108)])
def test_cloud_params_std140_offsets(field, offset):
    assert getattr(capi.CloudParamsGpu, field).offset == offset


@pytest.mark.parametrize("field,offset", [
    ("base_m", 0), ("top_m", 4), ("coverage", 8), ("density_scale", 12), ("cloud_type", 16),
    ("shape_bias", 20), ("detail_bias", 24), ("anvil_bias", 28), ("droplet_diameter_um", 32)])
def test_cloud_layer_offsets(field, offset):
    assert getattr(capi.CloudLayerGpu, field).offset == offset


@pytest.mark.parametrize("field,offset", [
    ("inv_view_proj", 192), ("camera_position_world", 256), ("sun_direction", 288),
    ("sun_illuminance", 304), ("viewport_size", 352), ("time_seconds", 368),
    ("simulated_seconds", 372), ("frame_index", 376), ("ev100", 380), ("prev_view_proj", 384)])
def test_frame_uniform_offsets(field, offset):
    assert getattr(capi.FrameUniformsGpu, field).offset == offset


def header_functions():
    text = (ROOT / "include" / "psclouds.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(psc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    names = header_functions()
    assert len(names) >= 30
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/psclouds.h but not exported"
    assert set(names) == set(capi.EXPORTED), set(names) ^ set(capi.EXPORTED)


def test_defaults_match_reference():
    p = capi.CloudParamsGpu()
    call("psc_params_default", C.byref(p))  # params.rs:142-212
    assert list(p.sigma_s) == pytest.approx([0.030, 0.040, 0.060])
    assert p.detail_strength == pytest.approx(0.05) and p.curl_strength == pytest.approx(0.1)
    assert (p.light_steps, p.cloud_steps, p.multi_scatter_octaves) == (6, 192, 4)
    assert (p.base_scale_m, p.detail_scale_m, p.weather_scale_m) == (4500.0, 800.0, 32000.0)
    assert p.wind_skew_strength == 0.5 and p.wind_drift_strength == 1.0
    w = capi.WorldUniformsGpu()
    call("psc_world_default", C.byref(w))  # weather.rs:60-84
    assert w.planet_radius_m == 6_360_000.0 and w.atmosphere_top_m == 6_460_000.0
    assert w.mie_g == pytest.approx(0.8)


def _ctx():
    c = C.c_void_p()
    call("psc_create", 0, C.byref(c))
    return c


def test_set_march_steps_clamps_like_reference():
    c = _ctx()  # lib.rs:709-712: cloud [8,256], light [1,16]
    try:
        call("psc_set_march_steps", c, 1000, 0)
        p = capi.CloudParamsGpu()
        call("psc_get_params", c, C.byref(p))
        assert (p.cloud_steps, p.light_steps) == (256, 1)
        call("psc_set_march_steps", c, 3, 99)
        call("psc_get_params", c, C.byref(p))
        assert (p.cloud_steps, p.light_steps) == (8, 16)
    finally:
        capi.lib().psc_destroy(c)


def _layer(base, top, t=0):
    return capi.CloudLayerGpu(base, top, 0.5, 1.0, t, 0.0, 0.0, 0.0, 20.0)


def test_layer_validation_errors():
    c = _ctx()
    try:
        ok = (capi.CloudLayerGpu * 2)(_layer(1500, 2300), _layer(4000, 5000))
        call("psc_set_layers", c, ok, 2)
        overlap = (capi.CloudLayerGpu * 2)(_layer(1000, 2000), _layer(1500, 2500))
        with pytest.raises(PscError) as e:
            call("psc_set_layers", c, overlap, 2)
        assert e.value.code == -3 and "overlap" in str(e.value)
        inverted = (capi.CloudLayerGpu * 1)(_layer(2000, 1000))
        with pytest.raises(PscError):
            call("psc_set_layers", c, inverted, 1)
        nine = (capi.CloudLayerGpu * 9)(*[_layer(1000 * i, 1000 * i + 500) for i in range(9)])
        with pytest.raises(PscError) as e:
            call("psc_set_layers", c, nine, 9)
        assert e.value.code == -3
        nan = (capi.CloudLayerGpu * 1)(_layer(float("nan"), 1000))
        with pytest.raises(PscError) as e:
            call("psc_set_layers", c, nan, 1)
        assert e.value.code == -2
        bad_type = (capi.CloudLayerGpu * 1)(_layer(1000, 2000, t=9))
        with pytest.raises(PscError):
            call("psc_set_layers", c, bad_type, 1)
    finally:
        capi.lib().psc_destroy(c)


def test_params_and_frame_validation_errors():
    c = _ctx()
    try:
        p = capi.CloudParamsGpu()
        call("psc_params_default", C.byref(p))
        p.base_scale_m = float("inf")
        with pytest.raises(PscError) as e:
            call("psc_set_params", c, C.byref(p))
        assert e.value.code == -2
        call("psc_params_default", C.byref(p))
        p.cloud_steps = 0
        with pytest.raises(PscError):
            call("psc_set_params", c, C.byref(p))
        f = capi.FrameUniformsGpu()
        w = capi.WorldUniformsGpu()
        call("psc_world_default", C.byref(w))
        f.sun_direction[1] = float("nan")
        with pytest.raises(PscError) as e:
            call("psc_set_frame", c, C.byref(f), C.byref(w))
        assert e.value.code == -2
        f.sun_direction[1] = 0.5
        f.frame_index = 0xFFFFFFFF  # a u32 whose bits are a NaN pattern is still valid
        call("psc_set_frame", c, C.byref(f), C.byref(w))
        w.atmosphere_top_m = w.planet_radius_m - 1
        with pytest.raises(PscError):
            call("psc_set_frame", c, C.byref(f), C.byref(w))
    finally:
        capi.lib().psc_destroy(c)


def test_render_without_inputs_is_an_error_not_a_crash():
    c = _ctx()
    try:
        v = capi.View(8, 8, None, None, None, None)
        with pytest.raises(PscError) as e:
            call("psc_render", c, C.byref(v), 1, None)
        assert e.value.code == -4  # MISSING_INPUT before any device work
        with pytest.raises(PscError):
            call("psc_render", None, C.byref(v), 1, None)
    finally:
        capi.lib().psc_destroy(c)


def test_options_validation():
    c = _ctx()
    try:
        o = capi.MarchOptions()
        call("psc_options_default", C.byref(o))
        call("psc_set_options", c, C.byref(o))
        o.storage = 9
        with pytest.raises(PscError):
            call("psc_set_options", c, C.byref(o))
        o.storage, o.filter = capi.STORAGE_BF16, capi.FILTER_TEXTURE
        with pytest.raises(PscError) as e:
            call("psc_set_options", c, C.byref(o))
        assert e.value.code == -8
        o.storage, o.schedule = capi.STORAGE_F16, capi.SCHED_PLAIN
        with pytest.raises(PscError) as e:
            call("psc_set_options", c, C.byref(o))
        assert e.value.code == -8
        o.schedule = capi.SCHED_FAST
        call("psc_set_options", c, C.byref(o))
    finally:
        capi.lib().psc_destroy(c)


def test_camera_frame_uniforms_match_numpy():
    cam = capi.FlyCamera((C.c_float * 3)(0.0, 100.0, 0.0), math.radians(10), math.radians(30),
                         0.0, math.radians(90), 0.1)
    f = capi.FrameUniformsGpu()
    call("psc_frame_from_camera", C.byref(cam), 320, 180, math.radians(35), math.radians(240),
         0.0047, 127500.0, C.byref(f))
    vp = np.array(f.view_proj, np.float64).T  # to row-major
    inv = np.array(f.inv_view_proj, np.float64).T
    assert np.allclose(inv @ vp, np.eye(4), atol=1e-5)
    # altaz_to_world (world.rs:110-114): +X east, +Y up, +Z south
    sun = np.array(f.sun_direction[:3])
    a, z = math.radians(35), math.radians(240)
    assert np.allclose(sun, [math.cos(a) * math.sin(z), math.sin(a), -math.cos(a) * math.cos(z)],
                       atol=1e-6)
    assert f.sun_illuminance[0] == 127500.0 and f.viewport_size[0] == 320.0
    # the view looks along FlyCamera::forward
    fwd = np.array([math.cos(math.radians(10)) * math.sin(math.radians(30)),
                    math.sin(math.radians(10)),
                    -math.cos(math.radians(10)) * math.cos(math.radians(30))])
    view = np.array(f.view, np.float64).T
    assert np.allclose(view[2, :3], -fwd, atol=1e-6)


def test_synthesise_layers_reports_overlap():
    d = (capi.CloudLayerDesc * 2)(capi.CloudLayerDesc(0, 1000, 2000, 0.5, -1, 0, 0, -1, -1),
                                  capi.CloudLayerDesc(1, 1500, 2500, 0.5, -1, 0, 0, -1, -1))
    out = (capi.CloudLayerGpu * 8)()
    with pytest.raises(PscError) as e:
        call("psc_synthesise_layers", d, 2, out)
    assert e.value.code == -3


def test_loaded_library_was_built_from_these_sources():
    """psc_build_id is the hash of the sources and flags the binary was
    compiled from; the one this process loaded must match the tree."""
    from pedalsky_b200 import build
    got = capi.lib().psc_build_id().decode()
    assert got == build.source_hash(), (got, build.source_hash())


def test_new_entry_points_validate_their_arguments_before_device_work():
    """The step tuner and the layer-parameter gradient reject bad arguments
    (and missing inputs) with an error code, without touching a GPU."""
    c = _ctx()
    try:
        views = (capi.BatchView * 1)()
        before, after = C.c_float(), C.c_float()
        for args in ((None, 1, 1e-3, 1e-3, 3), (views, 0, 1e-3, 1e-3, 3), (views, 1, 0.0, 1e-3, 3),
                     (views, 1, float("inf"), 1e-3, 3), (views, 1, 1e-3, 1.0, 3), (views, 1, 1e-3, -0.1, 3),
                     (views, 1, 1e-3, 1e-3, 0), (views, 1, 1e-3, 1e-3, 101)):
            with pytest.raises(PscError) as e:
                call("psc_autotune_steps", c, args[0], args[1], args[2], args[3], args[4], C.byref(before),
                     C.byref(after), None)
            assert e.value.code == -1, args
        v = capi.View(8, 8, None, None, None, None)
        g = (C.c_double * 6)()
        with pytest.raises(PscError) as e:
            call("psc_layer_param_gradient", c, C.byref(v), 0, None, None, g, None, None)
        assert e.value.code == -1
        bg = (C.c_float * 256)()
        with pytest.raises(PscError) as e:  # the context has no layers yet
            call("psc_layer_param_gradient", c, C.byref(v), 0, bg, bg, g, None, None)
        assert e.value.code == -1
    finally:
        capi.lib().psc_destroy(c)
