"""Host helper for the persistent batched march (`psc_render_batch`).

Builds the `PscBatchView` array for a list of `scenes.Scene` views, with
device buffers (torch, plumbing only) for depth, outputs and the HDR target.
"""
from __future__ import annotations

import ctypes as C

from . import capi, scenes
from .capi import call


class Batch:
    """Device buffers and the C view array of one batch."""

    def __init__(self, views: list, device, outputs=("hdr",), host_inputs=None):
        import torch
        self.views = views
        self.device = torch.device(device)
        self.arr = (capi.BatchView * len(views))()
        self.keep = []
        self.depth, self.bg, self.hdr, self.lum, self.trans = [], [], [], [], []
        for i, s in enumerate(views):
            if s.depth is not None:
                depth = torch.from_numpy(s.depth).to(self.device)
                bg = torch.from_numpy(s.background).to(self.device)
            else:
                depth, bg = scenes.device_inputs(s.frame, s.world, s.width, s.height, self.device)
            hdr = bg.clone() if "hdr" in outputs else None
            lum = (torch.zeros((s.height, s.width, 4), device=self.device)
                   if "luminance" in outputs else None)
            tr = (torch.zeros((s.height, s.width, 4), device=self.device)
                  if "transmittance" in outputs else None)
            v = self.arr[i]
            v.frame, v.params = s.frame, s.params
            for k in range(8):
                v.layers[k] = s.layers[k]
            v.n_layers, v.width, v.height = s.n_layers, s.width, s.height
            v.depth = depth.data_ptr()
            v.out_luminance = lum.data_ptr() if lum is not None else None
            v.out_transmittance = tr.data_ptr() if tr is not None else None
            v.hdr = hdr.data_ptr() if hdr is not None else None
            self.depth.append(depth)
            self.bg.append(bg)
            self.hdr.append(hdr)
            self.lum.append(lum)
            self.trans.append(tr)

    @property
    def rays(self) -> int:
        return sum(s.width * s.height for s in self.views)

    def reset_hdr(self):
        for h, b in zip(self.hdr, self.bg):
            if h is not None:
                h.copy_(b, non_blocking=True)

    def render(self, handle, stream=None):
        call("psc_render_batch", handle, self.arr, len(self.views),
             C.c_void_p(stream.cuda_stream if stream is not None else None))


def set_tuning(handle, threads=128, tile_w=16, use_graph=0, form=capi.BATCH_PERSISTENT):
    t = capi.BatchTuning(threads, tile_w, use_graph, form)
    call("psc_set_batch_tuning", handle, C.byref(t))


def autotune(handle, batch: Batch, reps=3, stream=None):
    best = capi.BatchTuning()
    ms = C.c_float()
    call("psc_autotune_batch", handle, batch.arr, len(batch.views), reps, C.byref(best),
         C.byref(ms), C.c_void_p(stream.cuda_stream if stream is not None else None))
    opts = capi.MarchOptions()
    call("psc_get_options", handle, C.byref(opts))
    return {"form": "per_view" if best.form == capi.BATCH_PER_VIEW else "persistent",
            "form_id": best.form, "threads": best.threads, "tile_w": best.tile_w,
            "tile_h": best.threads // 32 // (best.tile_w // 8) * 4,
            "light_batch": opts.light_batch, "ms": ms.value}


def autotune_steps(handle, batch: Batch, max_rel_err=1e-3, max_share=1e-3, reps=3, stream=None):
    """Lower each view's primary and light-march step counts while its image
    stays within `max_rel_err` (relative, composited over the view's hdr
    background) on all but `max_share` of its pixels (psc_autotune_steps).
    The chosen counts are written into the batch's view array; returns them
    with the batch's median time before and after."""
    before, after = C.c_float(), C.c_float()
    call("psc_autotune_steps", handle, batch.arr, len(batch.views), float(max_rel_err), float(max_share),
         int(reps), C.byref(before), C.byref(after),
         C.c_void_p(stream.cuda_stream if stream is not None else None))
    steps = [(batch.arr[i].params.cloud_steps, batch.arr[i].params.light_steps) for i in range(len(batch.views))]
    return {"steps": steps, "ms_before": before.value, "ms_after": after.value}
