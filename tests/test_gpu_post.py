"""GPU parity of the half-res and TAA forms (psc_render with options.half_res
/ options.taa, psc_taa_resolve, psc_composite_halfres) against the oracle's
restatement of the reference passes (oracle/oracle_post.py) on FP64-oracle
marches.  Same distribution bar as the full-res march tests."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle_post as OP
from pedalsky_b200 import capi, scenes
from pedalsky_b200.capi import PscError, call
from pedalsky_b200.subsystem import (CloudsTuning, PrepareContext, RenderContext, WeatherInputs,
                                     subsystem_for_scene)

from . import _gpu
from ._metrics import composite, rel_stats
from .test_gpu_march import _check

pytestmark = pytest.mark.gpu

SIZE = (384, 216)


def _torch():
    return _gpu.torch_cuda()


def _run(sub, scene, W, H, hdr_np=None, out_rt=True):
    """psc_render of one whole view; returns (rt_L, rt_T, hdr) as numpy."""
    torch = _torch()
    dev = torch.device("cuda", 0)
    rw, rh = C.c_uint32(), C.c_uint32()
    call("psc_cloud_rt_size", W, H, sub.options.half_res, C.byref(rw), C.byref(rh))
    L = torch.zeros((rh.value, rw.value, 4), device=dev)
    T = torch.zeros((rh.value, rw.value, 4), device=dev)
    depth = None if scene.depth is None else torch.from_numpy(scene.depth).to(dev)
    hdr = None if hdr_np is None else torch.from_numpy(np.ascontiguousarray(hdr_np, np.float32)).to(dev)
    v = capi.View(W, H, depth.data_ptr() if depth is not None else None,
                  L.data_ptr() if out_rt else None, T.data_ptr() if out_rt else None,
                  hdr.data_ptr() if hdr is not None else None)
    call("psc_render", sub.handle, C.byref(v), 1, None)
    torch.cuda.synchronize()
    return L.cpu().numpy(), T.cpu().numpy(), None if hdr is None else hdr.cpu().numpy()


def _opts(sub, **kw):
    o = capi.MarchOptions.from_buffer_copy(sub.options)
    for k, v in kw.items():
        setattr(o, k, v)
    sub.set_options(o)


@pytest.fixture(scope="module")
def halfres_ref(oracle, oracle_noise):
    s = scenes.precision_1080p(*SIZE)
    luts = oracle.bake_luts(s.frame, s.world)
    hs = OP.halfres_scene(s)
    L, T = oracle.render(hs, oracle_noise, luts)
    return s, luts, L, T


@pytest.mark.parametrize("sched,storage,filt", [("plain", "f32", "exact"), ("fast", "f16", "hybrid")])
def test_half_res_march_and_catmull_rom_composite(halfres_ref, oracle_noise, sched, storage, filt):
    s, luts, Lo, To = halfres_ref
    s.options.schedule = capi.SCHED_FAST if sched == "fast" else capi.SCHED_PLAIN
    s.options.storage = capi.STORAGE_NAMES[storage]
    s.options.filter = capi.FILTER_NAMES[filt]
    sub = subsystem_for_scene(s, luts=luts, noise=oracle_noise)
    _opts(sub, half_res=1, composite=1)
    W, H = SIZE
    L, T, hdr = _run(sub, s, W, H, hdr_np=s.background)
    sub.close()
    rw, rh = OP.half_res_size(W, H)
    assert L.shape == (rh, rw, 4)
    bg_rt = scenes.sky_background(OP.halfres_scene(s).frame, rw, rh)
    _check(f"halfres_rt/{sched}/{storage}/{filt}", composite(L, T, bg_rt), composite(Lo, To, bg_rt))
    ref = OP.composite_halfres(Lo, To, s.background)
    _check(f"halfres_composite/{sched}/{storage}/{filt}", hdr, ref)


@pytest.mark.parametrize("rw,rh,W,H", [(37, 21, 75, 43),   # the quad kernel, odd target edges
                                        (60, 40, 64, 48),   # more than half: the one-pixel kernel
                                        (96, 54, 64, 36)])  # an RT larger than its target
def test_composite_halfres_entry_point_matches_oracle(rw, rh, W, H):
    torch = _torch()
    rng = np.random.default_rng(5)
    L = rng.uniform(-100.0, 4000.0, (rh, rw, 4)).astype(np.float32)
    T = rng.uniform(-0.2, 1.2, (rh, rw, 4)).astype(np.float32)
    bg = rng.uniform(100.0, 9000.0, (H, W, 4)).astype(np.float32)
    d = [torch.from_numpy(a).cuda() for a in (L, T, bg)]
    call("psc_composite_halfres", d[0].data_ptr(), d[1].data_ptr(), rw, rh, d[2].data_ptr(), W, H, None)
    torch.cuda.synchronize()
    got = d[2].cpu().numpy()
    ref = OP.composite_halfres(L.astype(np.float64), T.astype(np.float64), bg.astype(np.float64))
    st = rel_stats(got, ref)
    # FP32 16-tap sums against FP64: the negative lobes cancel on random data
    assert st["p99"] < 1e-5 and st["max"] < 2e-4, st


def _two_frames(W, H, yaw2=0.6):
    """Frame 1, and frame 2 after a small turn with prev_view_proj = frame 1's."""
    f1 = scenes.frame_for(W, H)
    f2 = scenes.frame_for(W, H, yaw_deg=yaw2)
    for c in range(4):
        for r in range(4):
            f2.prev_view_proj[c][r] = f1.view_proj[c][r]
    return f1, f2


@pytest.fixture(scope="module")
def taa_ref(oracle, oracle_noise):
    """FP64 oracle marches of two frames at the half-res RT size, and the
    oracle TAA resolves (bootstrap, then 1/8 blend)."""
    W, H = SIZE
    s = scenes.precision_1080p(W, H)
    f1, f2 = _two_frames(W, H)
    out = {}
    hist = OP.TaaHistory()
    for k, f in ((1, f1), (2, f2)):
        s.frame = f
        hs = OP.halfres_scene(s)
        luts = oracle.bake_luts(hs.frame, hs.world)
        L, T = oracle.render(hs, oracle_noise, luts)
        rl, rt = hist.step(L, T, hs.frame)
        out[k] = (f, luts, L, T, rl, rt)
    return out


def test_taa_bootstrap_then_resolve_matches_oracle(taa_ref, oracle_noise):
    W, H = SIZE
    s = scenes.precision_1080p(W, H, storage=capi.STORAGE_F16, filt=capi.FILTER_HYBRID,
                               schedule=capi.SCHED_FAST)
    rw, rh = OP.half_res_size(W, H)
    bg_rt = None
    sub = None
    for k in (1, 2):
        f, luts, Lo, To, RLo, RTo = taa_ref[k]
        s.frame = f
        if sub is None:
            sub = subsystem_for_scene(s, luts=luts, noise=oracle_noise)
            _opts(sub, half_res=1, taa=1, composite=0)
        else:
            call("psc_set_frame", sub.handle, C.byref(f), C.byref(s.world))
            sub.set_atmosphere_luts(luts)
        L, T, _ = _run(sub, s, W, H)
        bg_rt = scenes.sky_background(OP.halfres_scene(s).frame, rw, rh)
        _check(f"taa_frame{k}", composite(L, T, bg_rt), composite(RLo, RTo, bg_rt))
        if k == 1:  # bootstrap: the resolve is the raw march (no clamp)
            _check("taa_frame1_is_march", composite(L, T, bg_rt), composite(Lo, To, bg_rt))
    sub.close()


def test_taa_pass_level_entry_equals_fused_form(oracle, oracle_noise):
    """psc_taa_resolve on the march output gives the same resolve as the
    fused psc_render TAA form, frame after frame; invalidation restarts."""
    torch = _torch()
    W, H = 96, 54
    s = scenes.precision_1080p(W, H, storage=capi.STORAGE_F16, filt=capi.FILTER_HYBRID,
                               schedule=capi.SCHED_FAST)
    f1, f2 = _two_frames(W, H, yaw2=1.0)
    luts = oracle.bake_luts(f1, s.world)
    fused = subsystem_for_scene(s, luts=luts, noise=oracle_noise)
    _opts(fused, taa=1)
    plain = subsystem_for_scene(s, luts=luts, noise=oracle_noise)
    dev = torch.device("cuda", 0)
    outs = []
    for f in (f1, f2, f2):
        for sub in (fused, plain):
            call("psc_set_frame", sub.handle, C.byref(f), C.byref(s.world))
        a = _run(fused, s, W, H)
        Lm, Tm, _ = _run(plain, s, W, H)  # march only
        cl, ct = torch.from_numpy(Lm).to(dev), torch.from_numpy(Tm).to(dev)
        ol, ot = torch.zeros_like(cl), torch.zeros_like(ct)
        call("psc_taa_resolve", plain.handle, cl.data_ptr(), ct.data_ptr(), W, H, ol.data_ptr(),
             ot.data_ptr(), None)
        torch.cuda.synchronize()
        assert np.array_equal(a[0], ol.cpu().numpy()) and np.array_equal(a[1], ot.cpu().numpy())
        outs.append((a[0], Lm))
    assert np.array_equal(outs[0][0], outs[0][1])      # bootstrap = march
    assert not np.array_equal(outs[1][0], outs[1][1])  # then history blends in
    call("psc_invalidate_taa_history", fused.handle)
    a = _run(fused, s, W, H)
    Lm, _, _ = _run(plain, s, W, H)
    assert np.array_equal(a[0], Lm)  # invalidated: bootstrap again
    fused.close()
    plain.close()


def test_taa_views_keep_separate_history(oracle, oracle_noise):
    W, H = 64, 36
    s = scenes.precision_1080p(W, H)
    luts = oracle.bake_luts(s.frame, s.world)
    sub = subsystem_for_scene(s, luts=luts, noise=oracle_noise)
    _opts(sub, taa=1)
    first0, _, _ = _run(sub, s, W, H)
    sub.set_active_view(1)
    first1, _, _ = _run(sub, s, W, H)
    assert np.array_equal(first0, first1)  # view 1 bootstraps on its own
    sub.set_active_view(7)                 # clamped to the last slot
    assert sub.active_view == 1
    sub.close()


def test_rt_forms_reject_what_they_cannot_do(oracle, oracle_noise):
    W, H = 32, 18
    s = scenes.precision_1080p(W, H)
    luts = oracle.bake_luts(s.frame, s.world)
    sub = subsystem_for_scene(s, luts=luts, noise=oracle_noise)
    _opts(sub, half_res=1)
    torch = _torch()
    buf = torch.zeros((H, W, 4), device="cuda")
    two = (capi.View * 2)(capi.View(W, H, None, buf.data_ptr(), None, None),
                          capi.View(W, H, None, buf.data_ptr(), None, None))
    with pytest.raises(PscError):
        call("psc_render", sub.handle, two, 2, None)
    sub_rect = capi.View(W // 2, H, None, buf.data_ptr(), None, None)
    sub_rect.viewport_w, sub_rect.viewport_h = W, H
    with pytest.raises(PscError):
        call("psc_render", sub.handle, C.byref(sub_rect), 1, None)
    sub.close()


def test_subsystem_mirror_runs_the_half_res_taa_passes(oracle, oracle_noise):
    """The three passes through the RenderSubsystem mirror with
    half_res_render + temporal_taa: the first frame composites the Catmull-Rom
    upsample of the raw half-res march."""
    torch = _torch()
    W, H = SIZE
    s = scenes.precision_1080p(W, H)
    luts = oracle.bake_luts(s.frame, s.world)
    hs = OP.halfres_scene(s)
    Lo, To = oracle.render(hs, oracle_noise, luts)
    ref = OP.composite_halfres(Lo, To, s.background)
    sub = subsystem_for_scene(s, luts=luts, noise=oracle_noise)
    t = CloudsTuning(cloud_steps=s.params.cloud_steps, light_steps=s.params.light_steps,
                     multi_scatter_octaves=s.params.multi_scatter_octaves,
                     detail_strength=s.params.detail_strength, half_res_render=True,
                     temporal_taa=True, wind_drift_strength=s.params.wind_drift_strength,
                     diurnal_strength=s.params.diurnal_strength)
    sub.reconfigure(t)
    sub.set_params(s.params)
    assert (sub.options.half_res, sub.options.taa) == (1, 1)
    color = torch.from_numpy(s.background).cuda()
    depth = torch.from_numpy(s.depth).cuda()
    ctx = RenderContext(color=color, depth=depth)
    for p in sub.register_passes():
        sub.dispatch_pass(p.id, ctx)
    torch.cuda.synchronize()
    _check("mirror_halfres_taa_frame1", color.cpu().numpy(), ref)
    t.freeze_time = True  # frozen time switches TAA off (lib.rs:776)
    sub.reconfigure(t)
    assert sub.options.taa == 0
    sub.close()
