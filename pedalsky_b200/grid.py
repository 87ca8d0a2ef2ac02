"""Host helper for the voxel-grid form of the march and its adjoint
(`psc_render_grid`, `psc_adjoint`).

Holds the device buffers of one grid problem (torch is plumbing for device
memory only): the grid values, background, target, L/T outputs, the
gradient grid and the two accumulated doubles (loss, d loss / d
density_scale).  Row bands of the viewport are views whose pointers start
at the band's first row, so several bands (or ranks) add into the same
gradient exactly as one full view does.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .capi import call


def density_grid(values, spec: dict) -> capi.DensityGrid:
    """PscDensityGrid over a device tensor of shape (ny, nz, nx)."""
    ny, nz, nx = values.shape
    return capi.DensityGrid(values.data_ptr(), nx, ny, nz, int(spec.get("checkpoint_every", 16)),
                            spec["min_x_m"], spec["min_z_m"], spec["size_x_m"], spec["size_z_m"],
                            spec["density_scale"], spec["exit_transmittance"])


class GridProblem:
    def __init__(self, scene, values, device="cuda:0", spec=None):
        import torch
        self.torch = torch
        self.scene = scene
        self.device = torch.device(device)
        self.spec = dict(scene.extra["grid_spec"] if spec is None else spec)
        self.values = torch.as_tensor(np.ascontiguousarray(values, np.float32)).to(self.device)
        h, w = scene.height, scene.width
        self.bg = torch.from_numpy(np.ascontiguousarray(scene.background, np.float32)).to(self.device)
        self.L = torch.zeros((h, w, 4), dtype=torch.float32, device=self.device)
        self.T = torch.zeros((h, w, 4), dtype=torch.float32, device=self.device)
        self.grad = torch.zeros_like(self.values)
        self.acc = torch.zeros(2, dtype=torch.float64, device=self.device)  # loss, d/d scale
        self.target = None

    def grid(self) -> capi.DensityGrid:
        return density_grid(self.values, self.spec)

    def set_target(self, target):
        t = self.torch.as_tensor(np.ascontiguousarray(target, np.float32) if isinstance(target, np.ndarray)
                                 else target)
        self.target = t.to(self.device).contiguous()

    def _view(self, rows=None, outputs=True):
        w, h = self.scene.width, self.scene.height
        r0, r1 = rows if rows else (0, h)
        off = r0 * w * 4 * 4  # bytes to the band's first row (float4 per pixel)
        v = capi.View(w, r1 - r0, None,
                      (self.L.data_ptr() + off) if outputs else None,
                      (self.T.data_ptr() + off) if outputs else None, None)
        if rows:
            v.viewport_w, v.viewport_h, v.x_offset, v.y_offset = w, h, 0, r0
        return v, off

    def render(self, handle, rows=None, stream=None):
        v, _ = self._view(rows)
        call("psc_render_grid", handle, C.byref(self.grid()), C.byref(v),
             C.c_void_p(stream.cuda_stream if stream is not None else None))
        return self.L, self.T

    def zero_grad(self):
        self.grad.zero_()
        self.acc.zero_()

    def adjoint(self, handle, rows=None, stream=None, outputs=True):
        """Adds this view's (or band's) loss and gradients into grad / acc."""
        assert self.target is not None, "set_target first"
        v, off = self._view(rows, outputs)
        acc = self.acc.data_ptr()
        call("psc_adjoint", handle, C.byref(self.grid()), C.byref(v),
             C.c_void_p(self.bg.data_ptr() + off), C.c_void_p(self.target.data_ptr() + off),
             C.c_void_p(self.grad.data_ptr()), C.c_void_p(acc + 8), C.c_void_p(acc),
             C.c_void_p(stream.cuda_stream if stream is not None else None))

    def layer_gradient(self, handle, out, rows=None, stream=None):
        """Adds d loss / d (base_m, top_m) of the layer for this view (or
        band) into `out`, a device float64 tensor of two values."""
        assert self.target is not None, "set_target first"
        v, off = self._view(rows, outputs=False)
        call("psc_layer_gradient", handle, C.byref(self.grid()), C.byref(v),
             C.c_void_p(self.bg.data_ptr() + off), C.c_void_p(self.target.data_ptr() + off),
             C.c_void_p(out.data_ptr()),
             C.c_void_p(stream.cuda_stream if stream is not None else None))
        return out

    def composite_image(self):
        """I = L + background * T (what the loss compares with the target)."""
        return self.L + self.bg * self.T
