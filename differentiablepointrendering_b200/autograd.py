"""The renderer as a differentiable torch operation.

``render(frame, params)`` returns the images of a :class:`DeviceFrame`'s
cameras for the surfel parameters ``params`` (the seven fields as CUDA
tensors in BVH order, as ``get_point_parameters`` orders them); its
backward pass is the renderer's adjoint.  Everything stays on the device,
on torch's current stream: the parameters are copied into the renderer
(``pale_apply_points_device``), the forward pass renders into the frame's
tensors, and the backward pass hands the incoming image gradient to the
adjoint as dL/dI and returns its per-surfel gradients.

The adjoint differentiates the radiance image (``output="raw"``, the
default).  ``output="ldr"`` returns the post-processed image and passes its
gradient to the adjoint unchanged, which is what Pale's training loop does
(python/training.py:625-662 feeds dL/d(LDR) to render_backward).  Which
gradient groups are non-zero follows the renderer's ``gradients`` setting
(opacity only, as the reference, or all seven).  Forward and backward draw
independent Monte Carlo samples, as render_forward and render_backward do.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Sequence

import torch

from . import _native as N
from .device import DeviceFrame
from .pale import _check
from .scene import POINT_FIELDS

FIELDS = POINT_FIELDS[:7]


def _points_struct(n: int, tensors: Sequence[torch.Tensor]) -> N.PalePoints:
    s = N.PalePoints()
    s.count = n
    for k, t in zip(FIELDS, tensors):
        setattr(s, k, C.cast(C.c_void_p(t.data_ptr()), N.f32p))
    return s


class _Render(torch.autograd.Function):
    @staticmethod
    def forward(ctx, frame: DeviceFrame, output: str, *params: torch.Tensor) -> torch.Tensor:
        r = frame.r
        n = r.num_points
        ps = [p.detach().contiguous() for p in params]
        for k, p in zip(FIELDS, ps):
            if not (p.is_cuda and p.dtype == torch.float32):
                raise ValueError(f"render: parameter '{k}' must be a float32 CUDA tensor")
        struct = _points_struct(n, ps)
        _check(r._lib, r._h, r._lib.pale_apply_points_device(r._h, C.byref(struct), frame._stream()),
               "apply_points_device")
        r._asset_stale = True
        frame.forward()
        ctx.frame = frame
        ctx.shapes = [p.shape for p in params]
        return (frame.ldr if output == "ldr" else frame.raw).clone()

    @staticmethod
    def backward(ctx, grad_image: torch.Tensor):
        frame: DeviceFrame = ctx.frame
        g = frame.backward(grad_image.contiguous())
        grads = [g[k].clone().reshape(shape) for k, shape in zip(FIELDS, ctx.shapes)]
        return (None, None, *grads)


def render(frame: DeviceFrame, params: Dict[str, torch.Tensor], output: str = "raw") -> torch.Tensor:
    """Packed (P, 4) image of the frame's cameras, differentiable in the
    seven parameter tensors of ``params`` (``frame.split`` gives the
    per-camera views)."""
    if output not in ("raw", "ldr"):
        raise ValueError("output must be 'raw' or 'ldr'")
    return _Render.apply(frame, output, *[params[k] for k in FIELDS])


def parameters(renderer, device=None, requires_grad: bool = True) -> Dict[str, torch.Tensor]:
    """The renderer's parameters (BVH order) as CUDA tensors, ready for a
    torch optimizer."""
    dev = torch.device(device or f"cuda:{torch.cuda.current_device()}")
    p = renderer.get_point_parameters()
    return {k: torch.tensor(p[k], device=dev, requires_grad=requires_grad) for k in FIELDS}
