"""ORACLE — test infrastructure, not product code.

NumPy (FP64) restatement of the two passes that sit between the cloud march
and the HDR target in the reference, for the parity tests of the half-res
and TAA forms:

  * half-res march set-up: cloud-RT size and the depth lookup of the patched
    march (crates/ps-clouds/src/lib.rs:746-758,
    crates/ps-clouds/src/pipeline.rs:277-319);
  * the 9-tap Catmull-Rom composite of a half-res cloud RT
    (shaders/clouds/cloud_composite_halfres.wgsl:60-126) with exact
    bilinear taps, clamp-to-edge, and the dual-source blend
    `dst = L + dst * T` (crates/ps-clouds/src/pipeline.rs:469-484);
  * the cloud TAA resolve (shaders/clouds/cloud_taa.wgsl:81-197) and the
    host's blend-weight / history bookkeeping (crates/ps-clouds/src/lib.rs:776-825).

Only tests/ import this module; it is the checker, never the thing measured.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from pedalsky_b200 import capi

HALF_RES_SCALE = 0.5          # crates/ps-clouds/src/lib.rs (HALF_RES_SCALE)
TAA_BLEND_WEIGHT = 1.0 / 8.0  # crates/ps-clouds/src/lib.rs:42


def half_res_size(width: int, height: int) -> tuple[int, int]:
    """Cloud-RT size: ((fb as f32 * 0.5) as u32).max(1) per axis (lib.rs:751-758)."""
    f = np.float32(HALF_RES_SCALE)
    return max(1, int(np.float32(width) * f)), max(1, int(np.float32(height) * f))


def halfres_depth(depth: np.ndarray, rw: int, rh: int) -> np.ndarray:
    """Depth seen by half-res RT pixel (x, y): the full-res texel at
    vec2<i32>(vec2<f32>(x, y) * (viewport / rt)) (pipeline.rs:296-305)."""
    h, w = depth.shape
    sx, sy = np.float32(w) / np.float32(rw), np.float32(h) / np.float32(rh)
    xs = (np.arange(rw, dtype=np.float32) * sx).astype(np.int64)
    ys = (np.arange(rh, dtype=np.float32) * sy).astype(np.int64)
    return np.ascontiguousarray(depth[ys[:, None], xs[None, :]], np.float32)


def halfres_scene(scene):
    """The half-res march is the full march of a frame whose viewport is the
    cloud RT (the patched shader divides fragment positions by the RT size
    for the view ray, the depth clip and the AP uv) with the depth read at
    the scaled position."""
    rw, rh = half_res_size(scene.width, scene.height)
    f = capi.FrameUniformsGpu.from_buffer_copy(scene.frame)
    f.viewport_size[0], f.viewport_size[1] = float(rw), float(rh)
    f.viewport_size[2], f.viewport_size[3] = 1.0 / rw, 1.0 / rh
    depth = None if scene.depth is None else halfres_depth(scene.depth, rw, rh)
    return dataclasses.replace(scene, width=rw, height=rh, frame=f, depth=depth, background=None)


def _bilinear_clamp(tex: np.ndarray, u: np.ndarray, v: np.ndarray) -> np.ndarray:
    """Exact bilinear sample of tex (h, w, c) at normalised (u, v), clamp to edge."""
    h, w = tex.shape[:2]
    x = u * w - 0.5
    y = v * h - 0.5
    x0, y0 = np.floor(x), np.floor(y)
    fx, fy = (x - x0)[..., None], (y - y0)[..., None]
    ix0 = np.clip(x0, 0, w - 1).astype(np.int64)
    ix1 = np.clip(x0 + 1, 0, w - 1).astype(np.int64)
    iy0 = np.clip(y0, 0, h - 1).astype(np.int64)
    iy1 = np.clip(y0 + 1, 0, h - 1).astype(np.int64)
    a = tex[iy0, ix0] * (1 - fx) + tex[iy0, ix1] * fx
    b = tex[iy1, ix0] * (1 - fx) + tex[iy1, ix1] * fx
    return a * (1 - fy) + b * fy


def catmull_rom_9_tap(tex: np.ndarray, out_w: int, out_h: int) -> np.ndarray:
    """catmull_rom_9_tap (cloud_composite_halfres.wgsl:60-100) evaluated at
    every output pixel centre uv = ((x + 0.5) / out_w, (y + 0.5) / out_h)."""
    t = np.asarray(tex, np.float64)
    th, tw = t.shape[:2]
    ux = (np.arange(out_w) + 0.5) / out_w
    uy = (np.arange(out_h) + 0.5) / out_h
    U, V = np.meshgrid(ux, uy)
    size = np.array([tw, th], np.float64)
    sp = np.stack([U, V], -1) * size
    tp1 = np.floor(sp - 0.5) + 0.5
    f = sp - tp1
    w0 = f * (-0.5 + f * (1.0 - 0.5 * f))
    w1 = 1.0 + f * f * (-2.5 + 1.5 * f)
    w2 = f * (0.5 + f * (2.0 - 1.5 * f))
    w3 = f * f * (-0.5 + 0.5 * f)
    w12 = w1 + w2
    off12 = w2 / np.maximum(w12, 1e-6)
    p0 = (tp1 - 1.0) / size
    p3 = (tp1 + 2.0) / size
    p12 = (tp1 + off12) / size
    px = (p0[..., 0], p12[..., 0], p3[..., 0])
    py = (p0[..., 1], p12[..., 1], p3[..., 1])
    wx = (w0[..., 0], w12[..., 0], w3[..., 0])
    wy = (w0[..., 1], w12[..., 1], w3[..., 1])
    out = np.zeros((out_h, out_w, t.shape[2]), np.float64)
    for j in range(3):
        for i in range(3):
            out += _bilinear_clamp(t, px[i], py[j]) * (wx[i] * wy[j])[..., None]
    return out


def composite_halfres(L_rt, T_rt, hdr):
    """Half-res composite over `hdr` (h, w, 4): Catmull-Rom upsample of the
    cloud RT, L >= 0, T in [0, 1], then dst = L + dst * T on all channels
    (cloud_composite_halfres.wgsl:110-126, blend One/Src1)."""
    h, w = hdr.shape[:2]
    L = np.maximum(catmull_rom_9_tap(L_rt, w, h), 0.0)
    T = np.clip(catmull_rom_9_tap(T_rt, w, h), 0.0, 1.0)
    return L + np.asarray(hdr, np.float64) * T


def _mat(m) -> np.ndarray:
    """glam column-major Mat4 ([col][row]) -> row-major numpy matrix."""
    return np.array([[m[c][r] for c in range(4)] for r in range(4)], np.float64)


def taa_resolve(cur_L, cur_T, hist_L, hist_T, frame, blend_weight, history_valid):
    """fs_main of cloud_taa.wgsl on a cloud RT of the current frame's size."""
    cur_L = np.asarray(cur_L, np.float64)
    cur_T = np.asarray(cur_T, np.float64)
    bw = min(max(float(blend_weight), 0.0), 1.0)
    if history_valid < 0.5 or bw >= 1.0:
        return cur_L.copy(), cur_T.copy()
    h, w = cur_L.shape[:2]
    U, V = np.meshgrid((np.arange(w) + 0.5) / w, (np.arange(h) + 0.5) / h)
    inv_vp, prev_vp = _mat(frame.inv_view_proj), _mat(frame.prev_view_proj)
    cam = np.array(frame.camera_position_world[:3], np.float64)
    ndc = np.stack([U * 2.0 - 1.0, 1.0 - V * 2.0, np.ones_like(U), np.ones_like(U)], -1)
    near_h = ndc @ inv_vp.T
    d = near_h[..., :3] / near_h[..., 3:4] - cam
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    clip = np.concatenate([d, np.zeros_like(d[..., :1])], -1) @ prev_vp.T
    ok = clip[..., 3] > 1e-4
    cw = np.where(ok, clip[..., 3], 1.0)
    pu = np.where(ok, (clip[..., 0] / cw) * 0.5 + 0.5, 0.0)
    pv = np.where(ok, 1.0 - ((clip[..., 1] / cw) * 0.5 + 0.5), 0.0)
    inside = ok & (pu >= 0.0) & (pv >= 0.0) & (pu <= 1.0) & (pv <= 1.0)
    hist_L = _bilinear_clamp(np.asarray(hist_L, np.float64), pu, pv)
    hist_T = _bilinear_clamp(np.asarray(hist_T, np.float64), pu, pv)

    def nbr_clamp(cur, hist):
        mn = np.full_like(cur, 1e10)
        mx = np.full_like(cur, -1e10)
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                ys = np.clip(np.arange(h) + dy, 0, h - 1)
                xs = np.clip(np.arange(w) + dx, 0, w - 1)
                s = cur[ys[:, None], xs[None, :]]
                mn, mx = np.minimum(mn, s), np.maximum(mx, s)
        return np.clip(hist, mn, mx)

    hL, hT = nbr_clamp(cur_L, hist_L), nbr_clamp(cur_T, hist_T)
    eb = np.where(inside, bw, 1.0)[..., None]
    L = np.maximum(hL * (1.0 - eb) + cur_L * eb, 0.0)
    T = np.clip(hT * (1.0 - eb) + cur_T * eb, 0.0, 1.0)
    return L, T


class TaaHistory:
    """Host bookkeeping of one view's TAA state (lib.rs:776-825): on the first
    active frame (or after invalidation / resize) the blend weight is 1 and
    history is not valid; afterwards 1/8 with valid history."""

    def __init__(self):
        self.valid = False
        self.L = self.T = None

    def step(self, cur_L, cur_T, frame):
        bw = TAA_BLEND_WEIGHT if self.valid else 1.0
        L, T = taa_resolve(cur_L, cur_T, self.L, self.T, frame, bw, 1.0 if self.valid else 0.0)
        self.L, self.T, self.valid = L, T, True
        return L, T
