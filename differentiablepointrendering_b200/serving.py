"""Serving: resident scenes, continuous admission and merged forward requests.

A :class:`Server` keeps every admitted scene's renderer resident on the GPU
(surfels, LBVH, photon-map and queue buffers stay allocated between
requests) and serves two kinds of request as they arrive:

* ``forward``: the LDR image of one camera;
* ``gradient``: the image, the L2 loss against a target image and the
  per-surfel gradients of that loss (forward with the fused loss, then the
  adjoint; the training loop's step 5-6 for one view).

Each scene has a worker thread, and each renderer runs on its own CUDA
stream, so requests for different scenes overlap on the device.  Within a
scene the worker takes every queued request when it becomes free: the
forward requests are merged into one render call over their cameras (one
wavefront over all of them, each camera rendered once however many
requests ask for it), then the gradient requests run one at a time (the
adjoint accumulates into one gradient array per scene, so gradient requests
cannot share a call).  Renderers are created with camera-keyed seeds
(``camera_seeds="camera"``), so a camera's image does not depend on which
other cameras share its call: a request gives the same result alone and in
the mix (gradients up to the order of float atomic additions).

Scenes are admitted against an HBM budget: ``add_scene`` measures the
device memory the new renderer holds after one forward and adjoint pass and
refuses the scene (:class:`AdmissionError`) if the admitted scenes would
exceed the budget.  Request latency is measured from ``submit`` to the
result being ready on the host.
"""
from __future__ import annotations

import ctypes as C
import threading
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import _native as N
from .pale import Renderer, _check
from .scene import SceneArrays


class AdmissionError(RuntimeError):
    """A scene does not fit the server's HBM budget."""


@dataclass
class Request:
    scene: str
    camera: int
    kind: str = "forward"                  # "forward" or "gradient"
    target: Optional[np.ndarray] = None    # gradient: (H, W, 3) target image
    # results, filled by the server
    image: Optional[np.ndarray] = None     # (H, W, 4) LDR
    loss: Optional[float] = None
    grads: Optional[Dict[str, np.ndarray]] = None   # BVH order
    error: Optional[str] = None
    batch_views: int = 0                   # cameras in the forward call that served it
    t_submit: float = 0.0
    t_done: float = 0.0
    done: threading.Event = field(default_factory=threading.Event, repr=False)

    @property
    def latency_ms(self) -> float:
        return (self.t_done - self.t_submit) * 1e3


def _device_used() -> int:
    import torch

    free, total = torch.cuda.mem_get_info()
    return int(total - free)


class _Scene:
    def __init__(self, name: str, renderer: Renderer, footprint: int, max_views: int):
        self.name = name
        self.r = renderer
        self.footprint = footprint
        self.max_views = max_views
        self.queue: List[Request] = []
        self.cv = threading.Condition()
        self.stop = False
        self.batches: List[int] = []
        self.thread = threading.Thread(target=self._run, name=f"pale-serve-{name}", daemon=True)

    # ------------------------------------------------------------ worker
    def _run(self):
        while True:
            with self.cv:
                while not self.queue and not self.stop:
                    self.cv.wait()
                if self.stop and not self.queue:
                    return
                reqs, self.queue = self.queue, []
            fwd = [q for q in reqs if q.kind == "forward"]
            grd = [q for q in reqs if q.kind == "gradient"]
            while fwd:
                cams = sorted({q.camera for q in fwd})[: self.max_views]
                now = [q for q in fwd if q.camera in cams]
                fwd = [q for q in fwd if q.camera not in cams]
                self._forward(cams, now)
            for q in grd:
                self._gradient(q)

    def _finish(self, q: Request):
        q.t_done = time.perf_counter()
        q.done.set()

    def _forward(self, cams: List[int], reqs: List[Request]):
        r = self.r
        try:
            pix = sum(r._sizes[i][0] * r._sizes[i][1] for i in cams)
            ldr = np.empty(pix * 4, np.float32)
            raw = np.empty(pix * 4, np.float32)
            idx = N.cams_array(cams)
            _check(r._lib, r._h, r._lib.pale_render_forward(r._h, len(cams), idx.ctypes.data_as(N.u32p),
                                                            ldr.ctypes.data_as(N.f32p), raw.ctypes.data_as(N.f32p)),
                   "serve forward")
            images, off = {}, 0
            for i in cams:
                w, h = r._sizes[i]
                images[i] = ldr[off:off + 4 * w * h].reshape(h, w, 4)
                off += 4 * w * h
            self.batches.append(len(cams))
            for q in reqs:
                q.image = images[q.camera].copy()
                q.batch_views = len(cams)
        except Exception as e:  # reported per request
            for q in reqs:
                q.error = str(e)
        for q in reqs:
            self._finish(q)

    def _gradient(self, q: Request):
        r = self.r
        try:
            name = r._names[q.camera]
            images, dldi, loss = r.render_forward_loss({name: np.asarray(q.target, np.float32)})
            grads, _ = r.render_backward(dldi)
            q.image, q.loss, q.grads = images[name], loss[name], grads
            q.batch_views = 1
        except Exception as e:
            q.error = str(e)
        self._finish(q)


class Server:
    """Resident scenes served by per-scene workers (see the module docs)."""

    def __init__(self, hbm_budget: int, max_views_per_call: int = 16):
        self.budget = int(hbm_budget)
        self.max_views = int(max_views_per_call)
        self.scenes: Dict[str, _Scene] = {}
        self.done: List[Request] = []
        self._lock = threading.Lock()

    @property
    def admitted_bytes(self) -> int:
        return sum(s.footprint for s in self.scenes.values())

    def add_scene(self, name: str, scene: SceneArrays, settings: Optional[dict] = None) -> int:
        """Makes `scene` resident if it fits the budget; returns the bytes it holds."""
        if name in self.scenes:
            raise ValueError(f"scene '{name}' is already resident")
        st = dict(settings or {})
        st["camera_seeds"] = "camera"
        before = _device_used()
        r = Renderer.from_scene(scene, st)
        try:
            # one forward and adjoint pass allocates what later requests use
            r.render_forward()
            name0 = r.get_camera_names()[0]
            w, h = r._sizes[0]
            r.render_backward({name0: np.zeros((h, w, 3), np.float32)})
            footprint = max(0, _device_used() - before)
        except Exception:
            r.close()
            raise
        if self.admitted_bytes + footprint > self.budget:
            r.close()
            raise AdmissionError(f"scene '{name}' needs {footprint / 2**30:.2f} GiB; "
                                 f"{(self.budget - self.admitted_bytes) / 2**30:.2f} GiB of the budget left")
        sc = _Scene(name, r, footprint, self.max_views)
        self.scenes[name] = sc
        sc.thread.start()
        return footprint

    def remove_scene(self, name: str):
        sc = self.scenes.pop(name)
        with sc.cv:
            sc.stop = True
            sc.cv.notify()
        sc.thread.join()
        sc.r.close()

    def submit(self, req: Request) -> Request:
        sc = self.scenes.get(req.scene)
        if sc is None:
            raise KeyError(f"scene '{req.scene}' is not resident")
        if req.kind not in ("forward", "gradient"):
            raise ValueError("kind must be 'forward' or 'gradient'")
        if not 0 <= req.camera < len(sc.r._names):
            raise IndexError("camera index out of range")
        if req.kind == "gradient" and req.target is None:
            raise ValueError("a gradient request needs a target image")
        req.t_submit = time.perf_counter()
        with sc.cv:
            sc.queue.append(req)
            sc.cv.notify()
        with self._lock:
            self.done.append(req)
        return req

    def latency(self, kind: Optional[str] = None) -> Dict[str, float]:
        """p50 / p99 / mean latency (ms) of the finished requests."""
        with self._lock:
            lat = [q.latency_ms for q in self.done if q.done.is_set() and (kind is None or q.kind == kind)]
        if not lat:
            return {"n": 0}
        a = np.asarray(lat)
        return {"n": int(a.size), "p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)),
                "mean": float(a.mean())}

    def close(self):
        for name in list(self.scenes):
            self.remove_scene(name)
