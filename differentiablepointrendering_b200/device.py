"""Device-resident rendering on CUDA tensors.

``DeviceFrame`` drives a :class:`~differentiablepointrendering_b200.pale.Renderer`
through the C-ABI's device entry points: images, dL/dI and gradients stay in
HBM as torch tensors and every kernel runs on the caller's CUDA stream, with
no host synchronisation.  Counters of a call are fetched on demand with
:meth:`stats`.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Sequence

import torch

from . import _native as N
from .pale import Renderer, _check
from .scene import POINT_FIELDS, POINT_WIDTH


class DeviceFrame:
    """Forward / adjoint passes of selected cameras into device tensors."""

    def __init__(self, renderer: Renderer, cameras: Optional[Sequence[int]] = None, device=None):
        self.r = renderer
        self.device = torch.device(device or f"cuda:{torch.cuda.current_device()}")
        self.cams = list(range(len(renderer.get_camera_names()))) if cameras is None else list(cameras)
        self._cams = N.cams_array(self.cams)
        self.sizes = [renderer._sizes[i] for i in self.cams]
        self.pixels = sum(w * h for w, h in self.sizes)
        f = dict(dtype=torch.float32, device=self.device)
        self.ldr = torch.zeros(self.pixels, 4, **f)
        self.raw = torch.zeros(self.pixels, 4, **f)
        self.dldi = torch.zeros(self.pixels, 4, **f)
        self.loss = torch.zeros(len(self.cams), dtype=torch.float64, device=self.device)
        n = renderer.num_points
        self.grads = {k: torch.zeros((n, POINT_WIDTH[k]) if POINT_WIDTH[k] > 1 else (n,), **f) for k in POINT_FIELDS}
        self._gstruct = N.PalePoints()
        self._gstruct.count = n
        for k in POINT_FIELDS:
            setattr(self._gstruct, k, C.cast(C.c_void_p(self.grads[k].data_ptr()), N.f32p))

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def forward(self):
        """Renders LDR and RAW images (packed (P, 4), camera after camera)."""
        L = self.r._lib
        rc = L.pale_render_forward_device(self.r._h, len(self.cams), self._cams.ctypes.data_as(N.u32p),
                                          C.c_void_p(self.ldr.data_ptr()), C.c_void_p(self.raw.data_ptr()),
                                          self._stream())
        _check(L, self.r._h, rc, "render_forward_device")
        return self.ldr, self.raw

    def forward_loss(self, target: torch.Tensor) -> torch.Tensor:
        """forward() with the L2 loss of every camera against `target`
        (packed (P, 3) or (P, 4), alpha ignored) computed by the
        post-process: dL/dI lands in self.dldi; returns the per-camera
        losses as a float64 device tensor (compute_l2_grad /
        compute_l2_loss, python/losses.py:10-45)."""
        t = target.contiguous()
        if t.dtype != torch.float32 or t.dim() != 2 or t.shape[0] != self.pixels or t.shape[1] not in (3, 4):
            raise ValueError(f"target must be float32 ({self.pixels}, 3 or 4)")
        L = self.r._lib
        rc = L.pale_render_forward_loss_device(self.r._h, len(self.cams), self._cams.ctypes.data_as(N.u32p),
                                               C.c_void_p(t.data_ptr()), t.shape[1],
                                               C.c_void_p(self.ldr.data_ptr()), C.c_void_p(self.raw.data_ptr()),
                                               C.c_void_p(self.dldi.data_ptr()), C.c_void_p(self.loss.data_ptr()),
                                               self._stream())
        _check(L, self.r._h, rc, "render_forward_loss_device")
        return self.loss

    def backward(self, dldi: Optional[torch.Tensor] = None):
        """Adjoint pass with packed dL/dI (P, 4) (alpha ignored); gradients
        land in self.grads (BVH order)."""
        d = self.dldi if dldi is None else dldi.contiguous()
        L = self.r._lib
        rc = L.pale_render_backward_device(self.r._h, len(self.cams), self._cams.ctypes.data_as(N.u32p),
                                           C.c_void_p(d.data_ptr()), C.byref(self._gstruct), self._stream())
        _check(L, self.r._h, rc, "render_backward_device")
        return self.grads

    def step(self, config: Optional[dict] = None, opacity_reset: Optional[float] = None):
        """Optimizer step from the gradients of the last backward, on this
        frame's stream (Renderer.optimizer_step)."""
        self.r.optimizer_step(config, opacity_reset, stream=self._stream())

    def split(self, packed: torch.Tensor) -> List[torch.Tensor]:
        """Packed (P, 4) -> list of (H, W, 4) views, one per camera."""
        out, off = [], 0
        for w, h in self.sizes:
            out.append(packed[off:off + w * h].view(h, w, 4))
            off += w * h
        return out

    def stats(self) -> Dict[str, float]:
        return self.r.stats()


def l2_grad_(dldi: torch.Tensor, ldr: torch.Tensor, target_rgb: torch.Tensor,
             sizes: Optional[Sequence[tuple]] = None) -> torch.Tensor:
    """dL/dI of L = 1/2 mean((I - T)^2) over the RGB values of each camera
    (compute_l2_grad, python/losses.py:28-45, applied per camera as
    training.py:634-657 does), written into dldi (P, 4) with torch ops.
    `sizes` lists the cameras' (W, H) in packing order (one camera if None);
    DeviceFrame.forward_loss does the same inside the post-process."""
    torch.sub(ldr[:, :3], target_rgb, out=dldi[:, :3])
    off = 0
    for w, h in (sizes or [(target_rgb.shape[0], 1)]):
        dldi[off:off + w * h, :3].div_(3 * w * h)
        off += w * h
    return dldi


class ViewBatch:
    """Views of several renderers (scenes) rendered together: the forward
    pass of every view is ONE camera-gather wavefront and the adjoint ONE
    wavefront of (view, pass) jobs, each path finding its scene through its
    view.  A view is (scene index, camera index, passes, depth): passes from
    1 to the scene's gather/adjoint passes, depth 0 (the scene's adjoint
    bounces) or fewer bounces.  Images, dL/dI and targets are packed in view
    order as DeviceFrame's; every call runs on the caller's CUDA stream with
    the wavefront buffers of the first renderer.  A view may carry a pass
    range as fifth and sixth entries (first pass, pass count; forward only):
    it then renders those passes of its passes, its running sums kept in
    the `partial` tensor of forward_loss between calls (a request rendered
    in slices over several batches)."""

    def __init__(self, renderers: Sequence[Renderer], views: Sequence[Sequence[int]], device=None):
        if not renderers:
            raise ValueError("no renderers")
        self.renderers = list(renderers)
        self.device = torch.device(device or f"cuda:{torch.cuda.current_device()}")
        vs = []
        for v in views:
            s, c, p, d, f, n = (list(v) + [0, 0, 0, 0, 0, 0])[:6]
            vs.append((int(s), int(c), int(p), int(d), int(f), int(n)))
        self.views = vs
        self.sliced = any(n for *_, n in vs)
        arr = (N.PaleView * max(1, len(vs)))()
        for i, (s, c, p, d, f, n) in enumerate(vs):
            if not 0 <= s < len(self.renderers):
                raise ValueError(f"view {i}: scene {s} outside the {len(self.renderers)} renderers")
            arr[i].scene, arr[i].camera, arr[i].passes, arr[i].depth = s, c, p, d
            arr[i].first_pass, arr[i].pass_count = f, n
        self._views = arr
        self._scenes = (C.c_void_p * len(self.renderers))(*[r._h.value for r in self.renderers])
        self.sizes = [self.renderers[v[0]]._sizes[v[1]] for v in vs]
        self.pixels = sum(w * h for w, h in self.sizes)
        f = dict(dtype=torch.float32, device=self.device)
        self.ldr = torch.zeros(max(1, self.pixels), 4, **f)
        self.raw = torch.zeros(max(1, self.pixels), 4, **f)
        self.dldi = torch.zeros(max(1, self.pixels), 4, **f)
        self.loss = torch.zeros(max(1, len(vs)), dtype=torch.float64, device=self.device)
        self.grads = []
        self._gstructs = (N.PalePoints * len(self.renderers))()
        for k, r in enumerate(self.renderers):
            n = r.num_points
            g = {key: torch.zeros((n, POINT_WIDTH[key]) if POINT_WIDTH[key] > 1 else (n,), **f) for key in POINT_FIELDS}
            self.grads.append(g)
            self._gstructs[k].count = n
            for key in POINT_FIELDS:
                setattr(self._gstructs[k], key, C.cast(C.c_void_p(g[key].data_ptr()), N.f32p))

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def forward_loss(self, target: Optional[torch.Tensor] = None, trace_photons: bool = True,
                     partial: Optional[torch.Tensor] = None):
        """Forward render of every view (with the L2 loss against `target`,
        packed (P, 3) or (P, 4), when given); returns the per-view losses
        (float64 device tensor) or None.  partial: packed (P, 4) running
        sums of the views rendered in slices (read for a view whose range
        starts after pass 0, written for a view not finished)."""
        L = self.renderers[0]._lib
        t = None
        if target is not None:
            t = target.contiguous()
            if t.dtype != torch.float32 or t.dim() != 2 or t.shape[0] != self.pixels or t.shape[1] not in (3, 4):
                raise ValueError(f"target must be float32 ({self.pixels}, 3 or 4)")
        rc = L.pale_render_views_loss_device(
            len(self.renderers), self._scenes, 1 if trace_photons else 0, len(self.views), self._views,
            C.c_void_p(t.data_ptr()) if t is not None else None, t.shape[1] if t is not None else 0,
            C.c_void_p(self.ldr.data_ptr()), C.c_void_p(self.raw.data_ptr()),
            C.c_void_p(self.dldi.data_ptr()) if t is not None else None,
            C.c_void_p(self.loss.data_ptr()) if t is not None else None,
            C.c_void_p(partial.data_ptr()) if partial is not None else None, self._stream())
        _check(L, self.renderers[0]._h, rc, "render_views_loss_device")
        return self.loss if t is not None else None

    def backward(self, dldi: Optional[torch.Tensor] = None):
        """Adjoint pass of every view with packed dL/dI (P, 4) (default: the
        last forward_loss's); returns one gradient dict per renderer (BVH
        order)."""
        d = self.dldi if dldi is None else dldi.contiguous()
        L = self.renderers[0]._lib
        rc = L.pale_render_views_backward_device(len(self.renderers), self._scenes, len(self.views), self._views,
                                                 C.c_void_p(d.data_ptr()), self._gstructs, self._stream())
        _check(L, self.renderers[0]._h, rc, "render_views_backward_device")
        return self.grads

    def view_gradients(self, views: Sequence[int], dldi: Optional[torch.Tensor] = None) -> List[Dict[str, torch.Tensor]]:
        """The gather estimator's backward of the last forward_loss (the
        first renderer's estimator must be "gather") with gradients per
        view: one gradient dict (BVH order of the view's scene) for each
        view index in `views`; the other views are not swept."""
        d = self.dldi if dldi is None else dldi.contiguous()
        f = dict(dtype=torch.float32, device=self.device)
        structs = (N.PalePoints * max(1, len(self.views)))()
        out = []
        for i in views:
            s = self.views[i][0]
            n = self.renderers[s].num_points
            g = {key: torch.empty((n, POINT_WIDTH[key]) if POINT_WIDTH[key] > 1 else (n,), **f) for key in POINT_FIELDS}
            out.append(g)
            structs[i].count = n
            for key in POINT_FIELDS:
                setattr(structs[i], key, C.cast(C.c_void_p(g[key].data_ptr()), N.f32p))
        L = self.renderers[0]._lib
        rc = L.pale_render_views_gradients_device(len(self.renderers), self._scenes, len(self.views), self._views,
                                                  C.c_void_p(d.data_ptr()), structs, self._stream())
        _check(L, self.renderers[0]._h, rc, "render_views_gradients_device")
        return out

    def split(self, packed: torch.Tensor) -> List[torch.Tensor]:
        """Packed (P, 4) -> list of (H, W, 4) views, one per view."""
        out, off = [], 0
        for w, h in self.sizes:
            out.append(packed[off:off + w * h].view(h, w, 4))
            off += w * h
        return out
