"""The density bound behind the FAST march's step skip, checked on the CPU.

The FAST march tests a primary step's profile before fetching any noise: the
reference's base shape remap(R, -(1 - lf), 1, 0, 1) is at most 1, the coverage
remap turns cloud into cloud - (1 - eff), and the detail erosion
remap(cloud, lo, 1, 0, 1) only lowers a cloud value <= 1, so the sample density
(cloud_march.wgsl:432-530) is at most clamp01(ndf(h) - (1 - eff)) * density_scale.
Steps whose bound is at or below the 1e-3 density threshold are skipped.
These tests evaluate the oracle's FP64 restatement of sample_density at random
points of every cloud type and check the bound.
"""
import numpy as np
import pytest

from oracle import pyoracle
from pedalsky_b200 import scenes


@pytest.fixture(scope="module")
def noise():
    return pyoracle.bake_noise()


def _points(rng, layer, planet_r, n):
    """n random world points inside the layer's shell within 15 km of the origin."""
    x = rng.uniform(-15000.0, 15000.0, n)
    z = rng.uniform(-15000.0, 15000.0, n)
    alt = rng.uniform(layer.base_m, layer.top_m, n)
    y = np.sqrt((planet_r + alt) ** 2 - x * x - z * z) - planet_r
    return np.stack([x, y, z], 1), alt


def _check_scene(scene, noise, n_per_layer, rng, weather_values, attained=False):
    luts = pyoracle.bake_luts(scene.frame, scene.world)
    R = scene.world.planet_radius_m
    n_layers = scene.params.cloud_layer_count
    dense = 0
    for li in range(n_layers):
        L = scene.layers[li]
        pts, alts = _points(rng, L, R, n_per_layer)
        for p3, alt, wr in zip(pts, alts, rng.choice(weather_values, n_per_layer)):
            d, prof = pyoracle.density_sample(scene, noise, luts, li, p3, alt, wr)
            eff = min(max(wr * L.coverage, 0.0), 1.0)
            # density = clamp01(cloud) * density_scale; the profile exceeds 1 in
            # the Cumulonimbus anvil
            bound = min(max(prof - (1.0 - eff), 0.0), 1.0) * L.density_scale if eff >= 0.01 else 0.0
            assert d <= bound * (1 + 1e-9) + 1e-12, (li, L.cloud_type, alt, wr, d, bound)
            h = (alt - L.base_m) / max(L.top_m - L.base_m, 1.0)
            if attained and h >= 0.1:
                assert d >= bound * (1 - 1e-9) - 1e-12, (li, L.cloud_type, alt, wr, d, bound)
            dense += d > 1e-3
    return dense


def test_bound_holds_on_the_three_layer_scene(noise):
    rng = np.random.default_rng(0)
    s = scenes.precision_1080p(64, 36)
    # the reference's synthesis writes R = 1; other values exercise the eff term
    dense = _check_scene(s, noise, 300, rng, np.array([1.0, 1.0, 0.8, 0.5, 0.05, 0.0]))
    assert dense > 50  # the check ran through dense samples, not only empty ones


def test_bound_holds_for_every_cloud_type(noise):
    rng = np.random.default_rng(1)
    s = scenes.precision_1080p(64, 36)
    s.params.diurnal_strength = 1.0  # shape/detail biases of the convective types
    for t in range(8):
        s.layers[0].cloud_type = t
        s.layers[0].anvil_bias = 1.5
        s.layers[0].shape_bias = 0.4
        s.layers[0].detail_bias = 0.3
        _check_scene(s, noise, 120, rng, np.array([1.0, 0.7]))


def test_bound_holds_on_the_cumulonimbus_stress_scene(noise):
    rng = np.random.default_rng(2)
    s = scenes.stress_2160p(64, 36)
    grid = s.weather.astype(np.float64)
    dense = _check_scene(s, noise, 400, rng, rng.choice(grid, 64))
    assert dense > 20


def test_bound_is_attained_with_saturated_noise(noise):
    """Base R = 255 everywhere makes the base shape exactly 1; detail = 255
    makes the erosion vanish for h >= 0.1.  There the density equals the
    bound, so the bound is the sharp one, not merely a true one."""
    sat = dict(noise)
    base = noise["base"].copy().reshape(-1, 4)
    base[:, 0] = 255
    sat["base"] = base.reshape(noise["base"].shape)
    sat["detail"] = np.full_like(noise["detail"], 255)
    rng = np.random.default_rng(3)
    s = scenes.precision_1080p(64, 36)
    dense = _check_scene(s, sat, 200, rng, np.array([1.0, 0.9, 0.6]), attained=True)
    assert dense > 100
    for t in range(8):
        s.layers[0].cloud_type = t
        s.layers[0].anvil_bias = 1.5
        _check_scene(s, sat, 60, rng, np.array([1.0, 0.7]), attained=True)
