"""CPU checks of the oracle's restatement of the half-res composite and the
cloud TAA (oracle/oracle_post.py) against independent formulations:
the 9-tap Catmull-Rom equals the textbook 16-tap kernel, reproduces
constants and linear ramps, and the TAA resolve obeys its defining
properties (bootstrap, identity reprojection, neighbourhood clamp)."""
import numpy as np
import pytest

from oracle import oracle_post as OP
from pedalsky_b200 import scenes


def _catmull_rom_16(tex, out_w, out_h):
    """Direct separable Catmull-Rom (B = 0, C = 0.5) over clamped indices."""
    th, tw = tex.shape[:2]

    def axis(n_out, n_src):
        sp = (np.arange(n_out) + 0.5) / n_out * n_src
        i1 = np.floor(sp - 0.5).astype(np.int64)
        f = sp - (i1 + 0.5)

        def k(x):  # Catmull-Rom kernel of distance x
            x = np.abs(x)
            return np.where(x < 1, 1.5 * x ** 3 - 2.5 * x ** 2 + 1,
                            np.where(x < 2, -0.5 * x ** 3 + 2.5 * x ** 2 - 4 * x + 2, 0.0))

        idx = np.stack([np.clip(i1 + d, 0, n_src - 1) for d in (-1, 0, 1, 2)], -1)
        wts = np.stack([k(f - d) for d in (-1, 0, 1, 2)], -1)
        return idx, wts

    ix, wx = axis(out_w, tw)
    iy, wy = axis(out_h, th)
    out = np.zeros((out_h, out_w, tex.shape[2]))
    for j in range(4):
        for i in range(4):
            out += tex[iy[:, j]][:, ix[:, i]] * (wy[:, j][:, None] * wx[:, i][None, :])[..., None]
    return out


@pytest.mark.parametrize("src,dst", [((8, 6), (16, 12)), ((7, 5), (15, 11)), ((3, 2), (6, 5)),
                                     ((1, 1), (2, 3))])
def test_nine_tap_equals_sixteen_tap(src, dst):
    rng = np.random.default_rng(3)
    tex = rng.uniform(-1, 2, (src[1], src[0], 4))
    a = OP.catmull_rom_9_tap(tex, *dst)
    b = _catmull_rom_16(tex, *dst)
    assert np.allclose(a, b, atol=1e-12, rtol=1e-12)


def test_catmull_rom_reproduces_constants_and_linear_ramps():
    c = np.full((9, 13, 4), 0.37)
    assert np.allclose(OP.catmull_rom_9_tap(c, 26, 18), 0.37, atol=1e-14)
    x = np.arange(13, dtype=np.float64)
    ramp = np.broadcast_to((2.0 * x + 1.0)[None, :, None], (9, 13, 1)).copy()
    up = OP.catmull_rom_9_tap(ramp, 26, 18)[..., 0]
    # interior output pixels (kernel support away from the clamped border)
    ux = (np.arange(26) + 0.5) / 26 * 13 - 0.5
    inner = (ux > 1.5) & (ux < 10.5)
    assert np.allclose(up[:, inner], (2.0 * ux[inner] + 1.0)[None, :], atol=1e-12)


def test_half_res_sizes_follow_the_reference():
    assert OP.half_res_size(1920, 1080) == (960, 540)
    assert OP.half_res_size(1921, 1079) == (960, 539)
    assert OP.half_res_size(1, 1) == (1, 1)
    assert OP.half_res_size(3, 5) == (1, 2)


def test_half_res_depth_reads_the_scaled_texel():
    d = np.arange(7 * 11, dtype=np.float32).reshape(7, 11)
    rw, rh = OP.half_res_size(11, 7)
    got = OP.halfres_depth(d, rw, rh)
    for y in range(rh):
        for x in range(rw):
            sx, sy = np.float32(11) / np.float32(rw), np.float32(7) / np.float32(rh)
            assert got[y, x] == d[int(np.float32(y) * sy), int(np.float32(x) * sx)]


def test_half_res_scene_is_a_march_at_the_rt_size():
    s = scenes.precision_1080p(64, 36)
    h = OP.halfres_scene(s)
    assert (h.width, h.height) == (32, 18)
    assert tuple(h.frame.viewport_size[:2]) == (32.0, 18.0)
    assert h.depth.shape == (18, 32)
    assert list(h.frame.inv_view_proj[0]) == list(s.frame.inv_view_proj[0])


def test_composite_halfres_clamps_before_blending():
    L = np.full((2, 2, 4), -5.0)
    T = np.full((2, 2, 4), 3.0)
    hdr = np.full((4, 4, 4), 2.0)
    out = OP.composite_halfres(L, T, hdr)
    assert np.allclose(out, 2.0)  # L -> 0, T -> 1


def _frames(yaw_deg=0.0):
    a = scenes.frame_for(40, 24)
    b = scenes.frame_for(40, 24, yaw_deg=yaw_deg)
    for c in range(4):
        for r in range(4):
            b.prev_view_proj[c][r] = a.view_proj[c][r]
    return a, b


def test_taa_bootstrap_returns_the_current_sample():
    rng = np.random.default_rng(0)
    cur_L, cur_T = rng.uniform(-1, 5, (24, 40, 4)), rng.uniform(-0.5, 1.5, (24, 40, 4))
    _, f = _frames()
    L, T = OP.taa_resolve(cur_L, cur_T, None, None, f, 1.0, 0.0)
    assert np.array_equal(L, cur_L) and np.array_equal(T, cur_T)  # no clamp on bootstrap
    hist = OP.TaaHistory()
    L2, T2 = hist.step(cur_L, cur_T, f)
    assert np.array_equal(L2, cur_L) and hist.valid


def test_taa_with_an_unmoved_camera_blends_toward_the_clamped_history():
    rng = np.random.default_rng(1)
    cur_L = rng.uniform(0, 5, (24, 40, 4))
    cur_T = rng.uniform(0, 1, (24, 40, 4))
    _, f = _frames(0.0)
    # history equal to the current frame: the resolve is the current frame
    L, T = OP.taa_resolve(cur_L, cur_T, cur_L, cur_T, f, OP.TAA_BLEND_WEIGHT, 1.0)
    assert np.allclose(L, cur_L, atol=1e-5) and np.allclose(T, cur_T, atol=1e-5)
    # a history far outside the neighbourhood is clamped to its AABB
    L2, _ = OP.taa_resolve(cur_L, cur_T, cur_L + 100.0, cur_T, f, OP.TAA_BLEND_WEIGHT, 1.0)
    assert np.all(L2 <= cur_L.max() + 1e-9)
    assert np.all(L2 >= cur_L - 1e-9)


def test_taa_reprojection_follows_a_camera_turn():
    """A 2 degree yaw shifts every pixel's history sample by the same
    sub-pixel amount (horizontal field of view ~118 degrees over 40 px), and
    an unmoved camera samples each pixel's own texel."""
    h, w = 24, 40
    ramp = np.broadcast_to(np.arange(w, dtype=np.float64)[None, :, None], (h, w, 4)).copy()
    # a current frame whose every 3x3 neighbourhood spans +-1e9, so the AABB
    # clamp lets the history through; weight 1e-12 keeps its trace negligible
    chk = np.where((np.add.outer(np.arange(h), np.arange(w)) % 2)[..., None] == 0, 1e9, -1e9)
    cur = np.broadcast_to(chk, (h, w, 4)).copy()
    shifts = {}
    for yaw in (0.0, 2.0):
        _, f = _frames(yaw)
        L, _ = OP.taa_resolve(cur, np.zeros_like(cur), ramp, np.zeros_like(cur), f, 1e-12, 1.0)
        d = (L[4:-4, 6:-6, 0] - ramp[4:-4, 6:-6, 0])
        shifts[yaw] = (float(np.median(d)), float(d.std()))
    assert abs(shifts[0.0][0]) < 1e-2
    assert 0.3 < abs(shifts[2.0][0]) < 1.2 and shifts[2.0][1] < 0.2, shifts
