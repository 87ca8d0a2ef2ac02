"""Helpers for the GPU tests: run a `scenes.Scene` through the C ABI."""
import ctypes as C

import numpy as np

from pedalsky_b200 import capi
from pedalsky_b200.capi import call, ptr
from pedalsky_b200.subsystem import subsystem_for_scene


def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU test without a CUDA device"
    return torch


def render(scene, noise=None, luts=None, sub=None, composite_bg=None, fused=False):
    """March `scene` on the GPU; returns (L, T) numpy (h, w, 4) and, with
    `composite_bg`, the composited HDR image as well."""
    torch = torch_cuda()
    own = sub is None
    if own:
        sub = subsystem_for_scene(scene, luts=luts, noise=noise)
    h, w = scene.height, scene.width
    dev = torch.device("cuda", 0)
    L = torch.zeros((h, w, 4), dtype=torch.float32, device=dev)
    T = torch.zeros((h, w, 4), dtype=torch.float32, device=dev)
    depth = None if scene.depth is None else torch.from_numpy(scene.depth).to(dev)
    hdr = None
    if composite_bg is not None:
        hdr = torch.from_numpy(np.ascontiguousarray(composite_bg, np.float32)).to(dev)
    if fused:
        o = capi.MarchOptions.from_buffer_copy(sub.options)
        o.composite = 1
        sub.set_options(o)
    view = capi.View(w, h, ptr(depth).value, L.data_ptr(), T.data_ptr(),
                     hdr.data_ptr() if (fused and hdr is not None) else None)
    stream = torch.cuda.current_stream().cuda_stream
    call("psc_render", sub.handle, C.byref(view), 1, C.c_void_p(stream))
    if hdr is not None and not fused:
        call("psc_composite", ptr(L), ptr(T), ptr(hdr), w, h, C.c_void_p(stream))
    torch.cuda.synchronize()
    out = (L.cpu().numpy(), T.cpu().numpy())
    if hdr is not None:
        out = out + (hdr.cpu().numpy(),)
    if own:
        sub.close()
    return out
