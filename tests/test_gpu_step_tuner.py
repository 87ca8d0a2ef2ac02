"""GPU tests of the step-count autotuner (`psc_autotune_steps`): it lowers a
view's light-march length and primary step count only while the view's
composited image stays within the bar against its render at the scene's own
counts, writes the chosen counts into the view array, and never touches the
views' own buffers.  The bar is checked here independently: the batch is
rendered again at the chosen counts and at the original ones, and the
relative error of L + background T (max over RGB) is measured in numpy."""
import numpy as np
import pytest

from pedalsky_b200 import batch as B
from pedalsky_b200 import capi, scenes
from pedalsky_b200.capi import PscError
from pedalsky_b200.subsystem import subsystem_for_scene

from . import _gpu

pytestmark = pytest.mark.gpu


def _views():
    kw = dict(storage=capi.STORAGE_F16, schedule=capi.SCHED_FAST, filt=capi.FILTER_HYBRID)
    return [scenes.precision_1080p(320, 180, **kw), scenes.precision_1080p(256, 144, steps=96, **kw)]


def _images(sub, views, counts, noise):
    b = B.Batch(views, "cuda:0", outputs=("luminance", "transmittance"))
    for i, (cs, ls) in enumerate(counts):
        b.arr[i].params.cloud_steps, b.arr[i].params.light_steps = cs, ls
    b.render(sub.handle)
    _gpu.torch_cuda().cuda.synchronize()
    return [(L.cpu().numpy(), T.cpu().numpy(), bg.cpu().numpy()) for L, T, bg in zip(b.lum, b.trans, b.bg)]


def _share_over(a, ref, thr):
    La, Ta, bg = a
    Lr, Tr, _ = ref
    I, Ir = La[..., :3] + bg[..., :3] * Ta[..., :3], Lr[..., :3] + bg[..., :3] * Tr[..., :3]
    r = (np.abs(I - Ir) / np.abs(Ir)).max(-1)
    return float((r > thr).mean())


def _next_down(c0, l0, c, l):
    """The tuner's next candidates past its choice (c, l): one light step
    less at the view's own primary count, and the next primary fraction at l."""
    nl = (c0, l - 1) if l > 1 and 2 * (l - 1) >= l0 else None
    fr = [max(8, (c0 * e + 7) // 8) for e in (7, 6, 5, 4)]
    below = [x for x in fr if x < c]
    nc = (below[0], l) if below else None
    return nl, nc


@pytest.mark.parametrize("max_rel_err", [1e-3, 2e-2, 2.5e-1])
def test_step_tuner_holds_its_bar_and_stops_at_its_edge(oracle_noise, max_rel_err):
    torch = _gpu.torch_cuda()
    views = _views()
    own = [(s.params.cloud_steps, s.params.light_steps) for s in views]
    sub = subsystem_for_scene(views[0], luts=None, noise=oracle_noise)
    try:
        b = B.Batch(views, "cuda:0", outputs=("hdr",))
        hdr_before = [h.clone() for h in b.hdr]
        res = B.autotune_steps(sub.handle, b, max_rel_err=max_rel_err, max_share=1e-3, reps=3)
        torch.cuda.synchronize()
        print(f"\n[step tuner {max_rel_err:g}] {own} -> {res['steps']}, "
              f"{res['ms_before']:.3f} -> {res['ms_after']:.3f} ms")
        # the views' own buffers are untouched
        for h0, h1 in zip(hdr_before, b.hdr):
            assert torch.equal(h0, h1)
        for (c0, l0), (c1, l1) in zip(own, res["steps"]):
            assert 8 <= c1 <= c0 and 1 <= l1 <= l0 and 2 * l1 >= l0 and 2 * c1 >= c0
        ref = _images(sub, views, own, oracle_noise)
        got = _images(sub, views, res["steps"], oracle_noise)
        # (the tuner counts on the GPU with fused multiply-adds, numpy without:
        # pixels right at the bar may fall either way, hence the 10 % slack)
        for g, r in zip(got, ref):
            assert _share_over(g, r, max_rel_err) <= 1.1e-3
        # each view's next reduction would have broken the bar
        for i, ((c0, l0), (c, l)) in enumerate(zip(own, res["steps"])):
            for nxt in _next_down(c0, l0, c, l):
                if nxt is None:
                    continue
                counts = list(res["steps"])
                counts[i] = nxt
                img = _images(sub, views, counts, oracle_noise)[i]
                share = _share_over(img, ref[i], max_rel_err)
                print(f"  view {i}: next {nxt} -> share over the bar {share:.2e}")
                assert share > 0.9e-3
        if max_rel_err >= 0.25:
            # a preview-quality bar lets the tuner cut steps, and fewer steps are faster
            assert all(s != o for s, o in zip(res["steps"], own))
            assert res["ms_after"] < res["ms_before"]
    finally:
        sub.close()


def test_step_tuner_argument_errors(oracle_noise):
    views = _views()
    sub = subsystem_for_scene(views[0], luts=None, noise=oracle_noise)
    try:
        b = B.Batch(views, "cuda:0", outputs=("hdr",))
        for kw in (dict(max_rel_err=0.0), dict(max_rel_err=float("nan")), dict(max_share=1.0), dict(reps=0)):
            with pytest.raises(PscError):
                B.autotune_steps(sub.handle, b, **kw)
    finally:
        sub.close()
