"""Host helper for the layer-parameter gradient of the procedural march
(`psc_layer_param_gradient`): d loss / d coverage, shape_bias, detail_bias,
density_scale, base_m and top_m of one scene layer, for the composite loss
of the grid adjoint (sum((L + background T - target)^2) / (3 viewport
pixels)).

Torch is plumbing for device memory only.  A view whose rectangle is a row
band of its viewport adds that band's share, so bands (or ranks) add up to
the whole image's gradient.
"""
from __future__ import annotations

import ctypes as C

from .capi import call
from .subsystem import _stream_handle

PARAMS = ("coverage", "shape_bias", "detail_bias", "density_scale", "base_m", "top_m")


def layer_param_gradient(handle, view, layer: int, background, target, grad, loss=None, stream=None) -> None:
    """Add d loss / d PARAMS of scene layer `layer` to `grad` (6 device
    doubles) and the loss to `loss` (1 device double, optional).
    `background` and `target` are device float32 tensors of shape
    (view.height, view.width, 4) covering the view's rectangle."""
    call("psc_layer_param_gradient", handle, C.byref(view), int(layer), C.c_void_p(background.data_ptr()),
         C.c_void_p(target.data_ptr()), C.c_void_p(grad.data_ptr()),
         C.c_void_p(loss.data_ptr()) if loss is not None else None, _stream_handle(stream))
