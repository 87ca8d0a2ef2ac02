"""CPU tests of the oracle itself: it reproduces its committed fixtures, its
own output moves under a one-ulp change of its inputs exactly where the march
sits on a branch margin, and it assembles the benchmark scenes without the
product library (the reference arm of bench.py depends on that)."""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from pedalsky_b200 import scenes

from ._metrics import composite

GOLDEN = Path(__file__).parent / "golden"
ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.parametrize("name", ["plain_96x54", "precision_96x54"])
def test_oracle_reproduces_committed_goldens(oracle, oracle_noise, name):
    """tests/golden/{plain,precision}_96x54.npz are FP64 renders of the plain
    and three-layer scenes; re-rendering them pins the restatement (and the
    input producers the scenes use) against drift."""
    s = scenes.plain_320x180(96, 54) if name == "plain_96x54" else scenes.precision_1080p(96, 54)
    luts = oracle.bake_luts(s.frame, s.world)
    L, T = oracle.render(s, oracle_noise, luts, precision=oracle.FP64)
    g = np.load(GOLDEN / f"{name}.npz")
    for got, want in ((L, g["L"]), (T, g["T"])):
        d = np.abs(got - want) / np.maximum(np.abs(want), 1e-30)
        assert d.max() <= 1e-6, float(d.max())


def _perturbed(width, height, sign_base, sign_top):
    """The three-layer scene with every layer's base and top moved by one
    FP32 ulp (0.1 mm at 1500 m, 1 mm at 9000 m)."""
    s = scenes.precision_1080p(width, height)
    for i in range(s.n_layers):
        b, t = np.float32(s.layers[i].base_m), np.float32(s.layers[i].top_m)
        s.layers[i].base_m = float(np.nextafter(b, np.float32(sign_base * 1e30)))
        s.layers[i].top_m = float(np.nextafter(t, np.float32(sign_top * 1e30)))
    return s


def test_fp64_oracle_flips_on_branch_margins(oracle, oracle_noise):
    """The FP64 march is only determined to within its branch flips: moving
    the layer altitudes by one FP32 ulp (the size of the rounding a FP32
    march makes in its sample positions) leaves 99.9 % of pixels within
    1e-4, but a few pixels move by more than 1e-3 — and each of those is a
    pixel whose march passes within 1e-3 of its early-exit threshold or 1e-2
    of its dense-sample threshold (oracle_branch_margins), which about 1 % of
    pixels do."""
    W, H = 480, 270
    s = scenes.precision_1080p(W, H)
    luts = oracle.bake_luts(s.frame, s.world)
    L, T = oracle.render(s, oracle_noise, luts, precision=oracle.FP64)
    ref = composite(L, T, s.background)
    mt, md = oracle.branch_margins(s, oracle_noise, luts)
    near = (mt < 1e-3) | (md < 1e-2)
    worst = np.zeros((H, W))
    for sb, st in ((1, 1), (-1, -1), (1, -1), (-1, 1)):
        p = _perturbed(W, H, sb, st)
        Lp, Tp = oracle.render(p, oracle_noise, luts, precision=oracle.FP64)
        img = composite(Lp, Tp, p.background)
        rel = (np.abs(img[..., :3] - ref[..., :3]) / np.abs(ref[..., :3])).max(-1)
        assert np.quantile(rel, 0.999) <= 1e-4
        worst = np.maximum(worst, rel)
    out = worst > 1e-3
    print(f"\n[oracle] one-ulp altitude change: {int(out.sum())} pixels above 1e-3, max "
          f"{worst.max():.2e}; pixels on a branch margin {near.mean():.3%}")
    assert out.sum() >= 1                 # the flips exist (max 4.0e-3 on this scene)
    assert (out & ~near).sum() == 0       # and every one is on a margin
    assert near.mean() < 0.03


def test_reference_arm_scene_assembly_maps_no_product_library():
    """With the oracle's restatements of the input producers
    (pyoracle.OracleHost), the benchmark scenes assemble without loading
    libpsclouds.so, and equal the library-assembled ones."""
    code = r"""
import sys
import numpy as np
sys.path.insert(0, %r)
from oracle import pyoracle
from pedalsky_b200 import capi, scenes
with scenes.host_helpers(pyoracle.OracleHost()):
    a = scenes.precision_1080p(96, 54)
    b = scenes.stress_2160p(96, 54, frame_index=5)
    g = scenes.grid_512(64, 64, grid_shape=(16, 8, 16))
maps = open("/proc/self/maps").read()
assert "libpsclouds" not in maps and capi._LIB is None, "product library mapped"
a2, b2 = scenes.precision_1080p(96, 54), scenes.stress_2160p(96, 54, frame_index=5)
for x, y in ((a, a2), (b, b2)):
    for f in ("params", "world", "options"):
        assert bytes(getattr(x, f)) == bytes(getattr(y, f)), f
    assert bytes(x.layers) == bytes(y.layers)
    assert np.allclose(np.array(x.frame.inv_view_proj), np.array(y.frame.inv_view_proj),
                       rtol=1e-6, atol=1e-9)
    assert np.array_equal(x.weather, y.weather) and np.array_equal(x.wind, y.wind)
print("ok")
""" % str(ROOT)
    res = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0 and "ok" in res.stdout, res.stdout + res.stderr
