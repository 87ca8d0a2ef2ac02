"""GPU test of `psc_render_batch_noalloc`, the batched march that allocates
no device memory when called.

It exists for callers that cannot call cudaMalloc while rendering: a frame
loop in which an allocation or free would synchronise the device, an engine
that owns a fixed device-memory budget, code running in a host callback.
Its work list lives in one fixed file-scope device array instead of
context-owned buffers, so this test checks that it draws the same images as
`psc_render_batch` (same kernel, same per-view LUT bakes) on two calls in a
row and on a non-default stream, that calls after the first leave free device
memory and the caching allocator's reservation unchanged, and that it refuses
what it cannot do without allocating, and a stream that is being captured
(its staging is shared by all calls).

The file name puts it last in collection order: it must pass both on its
own in a fresh process (where its first call also resolves the array's
device address) and after every other GPU test has used the library.
"""
import ctypes as C

import numpy as np
import pytest

from pedalsky_b200 import batch as B
from pedalsky_b200 import capi, scenes
from pedalsky_b200.capi import PscError, call
from pedalsky_b200.subsystem import subsystem_for_scene

from . import _gpu

pytestmark = pytest.mark.gpu

SKY_TEXELS = 192 * 108       # sky-view LUT texels per view
AP_TEXELS = 32 * 32 * 64     # aerial-perspective LUT texels per view
RTOL = 2e-6                  # the batched-march tolerance used against single-view renders
MAX_VIEWS = 64               # PSC_NOALLOC_MAX_VIEWS


def _noalloc(handle, batch, n, sky, ap, stream=None):
    call("psc_render_batch_noalloc", handle, batch.arr, n, C.c_void_p(sky.data_ptr()),
         C.c_void_p(ap.data_ptr()), C.c_void_p(stream.cuda_stream if stream is not None else None))


def _worst(got, want):
    worst = 0.0
    for (L, T), (L1, T1) in zip(zip(got.lum, got.trans), want):
        L, T = L.cpu().numpy(), T.cpu().numpy()
        assert np.isfinite(L).all() and np.isfinite(T).all()
        d = np.abs(L - L1)[..., :3] / np.maximum(np.abs(L1[..., :3]), 1.0)
        worst = max(worst, float(d.max()), float(np.abs(T - T1).max()))
    return worst


def _poison(batch):
    for L, T in zip(batch.lum, batch.trans):
        L.fill_(float("nan"))
        T.fill_(float("nan"))


def test_noalloc_batch_matches_render_batch_on_two_calls(oracle_noise):
    torch = _gpu.torch_cuda()
    dev = torch.device("cuda", 0)
    views = scenes.batch_views(10, seed=11, size_scale=0.06, storage=capi.STORAGE_F16,
                               filt=capi.FILTER_HYBRID)
    n = len(views)
    sub = subsystem_for_scene(views[0], luts=None, noise=oracle_noise)
    try:
        ref = B.Batch(views, dev, outputs=("luminance", "transmittance"))
        got = B.Batch(views, dev, outputs=("luminance", "transmittance"))
        sky = torch.empty(n * SKY_TEXELS * 4, dtype=torch.float32, device=dev)
        ap = torch.empty(n * AP_TEXELS * 4, dtype=torch.float32, device=dev)

        # No render has built the F16 noise storage or the texture objects
        # yet, and building them would allocate: the call must refuse.
        with pytest.raises(PscError) as e:
            _noalloc(sub.handle, got, n, sky, ap)
        assert e.value.code == -4

        ref.render(sub.handle)  # the allocating entry point; also builds the storage form
        torch.cuda.synchronize()
        want = [(L.cpu().numpy(), T.cpu().numpy()) for L, T in zip(ref.lum, ref.trans)]

        for k in range(2):
            _poison(got)
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info(dev)[0]
            _noalloc(sub.handle, got, n, sky, ap)
            torch.cuda.synchronize()
            free_after = torch.cuda.mem_get_info(dev)[0]
            if k == 1:  # the first call may load the library's GPU code for the array
                assert free_after == free_before, (free_before, free_after)
            worst = _worst(got, want)
            assert worst <= RTOL, (k, worst)

        # later calls, one of them on a non-default stream, allocate nothing:
        # device free memory and torch's reservation stay where they were
        side = torch.cuda.Stream(device=dev)
        reserved = torch.cuda.memory_reserved(dev)
        free0 = torch.cuda.mem_get_info(dev)[0]
        for k in range(3):
            _poison(got)
            torch.cuda.synchronize()
            _noalloc(sub.handle, got, n, sky, ap, stream=side if k == 1 else None)
            torch.cuda.synchronize()
            assert torch.cuda.mem_get_info(dev)[0] == free0, k
            assert torch.cuda.memory_reserved(dev) == reserved, k
            worst = _worst(got, want)
            assert worst <= RTOL, ("repeat", k, worst)
    finally:
        sub.close()


def test_noalloc_batch_refuses_a_capturing_stream(oracle_noise):
    """A graph recorded from this call would replay whatever the latest call
    staged, so a stream under capture is refused before anything is
    enqueued; the capture itself stays valid and ends empty."""
    torch = _gpu.torch_cuda()
    dev = torch.device("cuda", 0)
    views = scenes.batch_views(2, seed=5, size_scale=0.04, storage=capi.STORAGE_F16,
                               filt=capi.FILTER_HYBRID)
    sub = subsystem_for_scene(views[0], luts=None, noise=oracle_noise)
    try:
        b = B.Batch(views, dev, outputs=("luminance",))
        b.render(sub.handle)  # builds the storage form (allocating entry point)
        sky = torch.empty(2 * SKY_TEXELS * 4, dtype=torch.float32, device=dev)
        ap = torch.empty(2 * AP_TEXELS * 4, dtype=torch.float32, device=dev)
        _noalloc(sub.handle, b, 2, sky, ap)  # resolves the array's address outside the capture
        torch.cuda.synchronize()
        side = torch.cuda.Stream(device=dev)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(side):
            g.capture_begin(capture_error_mode="thread_local")
            try:
                with pytest.raises(PscError) as e:
                    _noalloc(sub.handle, b, 2, sky, ap, stream=side)
            finally:
                g.capture_end()
        assert e.value.code == -8 and "graph" in str(e.value)
        torch.cuda.synchronize()
        del g
    finally:
        sub.close()


def test_noalloc_batch_rejects_what_exceeds_its_array(oracle_noise):
    torch = _gpu.torch_cuda()
    dev = torch.device("cuda", 0)
    views = scenes.batch_views(2, seed=3, size_scale=0.04, storage=capi.STORAGE_F16,
                               filt=capi.FILTER_HYBRID)
    sub = subsystem_for_scene(views[0], luts=None, noise=oracle_noise)
    try:
        b = B.Batch(views, dev, outputs=("luminance",))
        sky = torch.empty(MAX_VIEWS * SKY_TEXELS * 4, dtype=torch.float32, device=dev)
        ap = torch.empty(MAX_VIEWS * AP_TEXELS * 4, dtype=torch.float32, device=dev)
        # more views than the array holds
        many = (capi.BatchView * (MAX_VIEWS + 1))(*[b.arr[i % 2] for i in range(MAX_VIEWS + 1)])
        with pytest.raises(PscError) as e:
            call("psc_render_batch_noalloc", sub.handle, many, MAX_VIEWS + 1,
                 C.c_void_p(sky.data_ptr()), C.c_void_p(ap.data_ptr()), None)
        assert e.value.code == -1 and "limit" in str(e.value)
        # more tiles than the array holds: a 32768 x 32768 view is 8 M tiles
        # of 16 x 8 pixels (rejected before anything is read or launched)
        b.arr[0].width = b.arr[0].height = 32768
        with pytest.raises(PscError) as e:
            _noalloc(sub.handle, b, 1, sky, ap)
        assert e.value.code == -1 and "limit" in str(e.value)
        # misaligned LUT buffer
        b.arr[0].width, b.arr[0].height = views[0].width, views[0].height
        with pytest.raises(PscError) as e:
            call("psc_render_batch_noalloc", sub.handle, b.arr, 1, C.c_void_p(sky.data_ptr() + 4),
                 C.c_void_p(ap.data_ptr()), None)
        assert e.value.code == -1
    finally:
        sub.close()
