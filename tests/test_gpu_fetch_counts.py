"""GPU test of psc_count_fetches, the instrumented build of the FAST kernel
that counts the fetches it issues (the measured side of the benchmark's
fetch roofline): it draws the same image as the timed kernel, and its counts
agree with the FP64 oracle's count of the same march's work."""
import ctypes as C

import numpy as np
import pytest

from pedalsky_b200 import capi, scenes
from pedalsky_b200.capi import PscError, call

from . import _gpu

pytestmark = pytest.mark.gpu


def _render_and_count(scene, count):
    torch = _gpu.torch_cuda()
    from pedalsky_b200.subsystem import subsystem_for_scene
    dev = torch.device("cuda", 0)
    sub = subsystem_for_scene(scene, luts=None)
    try:
        W, H = scene.width, scene.height
        L = torch.zeros((H, W, 4), dtype=torch.float32, device=dev)
        T = torch.zeros_like(L)
        depth = torch.from_numpy(scene.depth).to(dev)
        view = capi.View(W, H, depth.data_ptr(), L.data_ptr(), T.data_ptr(), None)
        fc = capi.FetchCounts()
        if count:
            call("psc_count_fetches", sub.handle, C.byref(view), C.byref(fc), None)
        else:
            call("psc_render", sub.handle, C.byref(view), 1, None)
        torch.cuda.synchronize()
        return L.cpu().numpy(), T.cpu().numpy(), fc.as_dict()
    finally:
        sub.close()


@pytest.mark.parametrize("storage,filt", [("f16", "hybrid"), ("u8", "exact")])
def test_fetch_counts_match_the_timed_kernel_and_the_oracle(oracle, oracle_noise, storage, filt):
    kw = dict(storage=capi.STORAGE_NAMES[storage], schedule=capi.SCHED_FAST,
              filt=capi.FILTER_NAMES[filt])
    s = scenes.precision_1080p(480, 270, **kw)
    L0, T0, _ = _render_and_count(s, count=False)
    L1, T1, c = _render_and_count(s, count=True)
    # the instrumented build computes the same image
    assert np.abs(L1 - L0).max() <= 1e-6 * max(np.abs(L0).max(), 1.0)
    assert np.abs(T1 - T0).max() <= 1e-6
    luts = oracle.bake_luts(s.frame, s.world)
    _, _, oc = oracle.render(s, oracle_noise, luts, precision=oracle.FP64, counters=True)
    print(f"\n[fetch counts] {storage}/{filt}: kernel {c}\n  oracle {oc}")
    n = s.width * s.height
    assert c["rays"] == n and c["depth_loads"] == n
    # the kernel runs only the steps of each layer whose altitude can pass
    # the profile test, so it executes fewer steps than the reference
    # algorithm, and the same dense samples (branch flips move a handful)
    assert c["live_steps"] <= c["primary_steps"] <= oc["steps"]
    assert abs(c["dense_samples"] - oc["dense"]) <= 1e-3 * oc["dense"]
    # the fetches the kernel proves unnecessary are skipped: a uniform
    # weather map is not sampled, and steps whose profile bound keeps them
    # below the density threshold fetch nothing
    assert c["weather_taps"] == 0 and c["type_loads"] == 0
    assert oc["dense"] <= c["live_steps"] + 1e-3 * oc["dense"] and c["live_steps"] < oc["base"]
    assert c["detail_taps"] <= c["live_steps"]
    # a warp's light march stops after 2 or 4 taps once every later tap of
    # every lane lies above the layer's last height of non-zero density
    assert 2 * c["dense_samples"] <= c["light_taps"] <= 6 * c["dense_samples"]
    assert c["skyview_taps"] == c["dense_samples"]
    assert c["transmittance_taps"] <= c["dense_samples"]
    assert abs(c["ap_taps"] - oc["ap"]) <= 1e-3 * max(oc["ap"], 1) + 2
    # every dense lane is counted in exactly one warp pass through the body
    assert c["dense_warp_lanes"] == c["dense_samples"]
    assert 0 < c["dense_warp_passes"] <= c["dense_samples"]
    print(f"  dense-body SIMT efficiency {c['dense_warp_lanes'] / (32 * c['dense_warp_passes']):.3f}")


def test_fetch_counts_reject_unsupported_forms(oracle_noise):
    s = scenes.precision_1080p(64, 36, storage=capi.STORAGE_F32, schedule=capi.SCHED_PLAIN)
    with pytest.raises(PscError) as e:
        _render_and_count(s, count=True)
    assert e.value.code == -8
