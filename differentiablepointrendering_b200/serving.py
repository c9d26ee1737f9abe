"""Serving: resident scenes and continuous batching of render requests.

A :class:`Server` keeps every admitted scene resident on the GPU: its
surfels, LBVH and photon map are built once when the scene is admitted and
stay in HBM between requests (the photon map is traced once, at admission,
as a scene that does not change needs no other).  Two kinds of request:

* ``forward``: the LDR image of one camera of a scene;
* ``gradient``: the image, the L2 loss against a target image and the
  per-surfel gradients of that loss (the training loop's forward with the
  fused loss, then the adjoint, for one view).

Each request carries its own number of passes (samples per pixel, gather
and adjoint) and adjoint bounces, up to the maxima its scene was created
with; resolutions are the scene's cameras.

Gradients: with the server's settings' estimator "reference" (default) the
round's gradient requests share adjoint wavefronts of the reference's
adjoint; with "gather" each gets the exact derivative of its view of the
round's forward (photon map held), swept from that forward's own path
vertices into arrays of its own (``pale_render_views_gradients_device``),
with no second wavefront.  The server's settings' ``gradients`` picks the
groups: opacity (default, as the reference's adjoint) or "all" seven; a
request's ``grads`` holds those only.

One dispatcher thread owns the GPU stream and serves requests in rounds.
A round takes the queued requests that fit (at most ``max_views`` views,
``max_pixels`` camera pixels, seven scenes and, when set, ``max_paths``
camera paths of pixels x passes, which bounds a round's time), in arrival
order or, with ``policy="light_first"``, the lightest first with requests
waiting longer than ``starve_s`` ahead of them (a request's weight: its
camera paths times its view's surfel layers per path, measured for every
camera when its scene is admitted), and renders them
together: the views of all the round's requests, of any scenes, are ONE
camera-gather wavefront (device.ViewBatch's entry point,
``pale_render_views_loss_device``), and the round's gradient requests share
ONE adjoint wavefront (``pale_render_views_backward_device``, up to eight
requests per wavefront) in which every request's gradients go to arrays of
its own.  Requests that arrive while a round runs are admitted to the next
round, as view slots and memory free up: continuous batching at round
granularity.

Seeds are keyed by camera (``camera_seeds="camera"``) and the photon maps
do not change, so a request's image and loss are the same alone and in any
mix, bit for bit, and its gradients up to the order of float atomic
additions.

Admission: ``add_scene`` measures the device memory the scene's renderer
holds (surfels, LBVH, photon map and grid, photon queues) and refuses the
scene (:class:`AdmissionError`) when the admitted scenes would exceed the
HBM budget.  The wavefront buffers shared by all rounds belong to a small
executor renderer of the server, sized by ``max_pixels`` on the first round.
Latency is measured from ``submit`` to the result being ready on the host.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from .pale import Renderer
from .scene import POINT_FIELDS, SceneArrays, make_box_scene


class AdmissionError(RuntimeError):
    """A scene does not fit the server's HBM budget."""


@dataclass
class Request:
    scene: str
    camera: int
    kind: str = "forward"                  # "forward" or "gradient"
    target: Optional[np.ndarray] = None    # gradient: (H, W, 3) target image
    passes: int = 0                        # samples per pixel (0: the scene's maximum)
    depth: int = 0                         # adjoint bounces (0: the scene's maximum)
    # results, filled by the server
    image: Optional[np.ndarray] = None     # (H, W, 4) LDR
    loss: Optional[float] = None
    # BVH order; the groups the server computes: opacity, or every field
    # when its settings ask for gradients="all"
    grads: Optional[Dict[str, np.ndarray]] = None
    error: Optional[str] = None
    batch_views: int = 0                   # views in the round that served it
    round: int = -1
    slices: int = 0                        # rounds its passes were rendered in
    t_submit: float = 0.0
    t_done: float = 0.0
    done: threading.Event = field(default_factory=threading.Event, repr=False)
    # server state: passes rendered so far, passes of the current round (0:
    # all that remain), running sums of a forward rendered in slices
    next_pass: int = field(default=0, repr=False)
    round_passes: int = field(default=0, repr=False)
    partial: object = field(default=None, repr=False)

    @property
    def latency_ms(self) -> float:
        return (self.t_done - self.t_submit) * 1e3


def _device_used() -> int:
    import torch

    free, total = torch.cuda.mem_get_info()
    return int(total - free)


@dataclass
class _Scene:
    name: str
    renderer: Renderer
    footprint: int
    max_passes: int
    max_depth: int
    layers: List[float] = field(default_factory=list)   # surfel layers per camera path, per camera


MAX_ROUND_SCENES = 7   # a call's scene table holds 8 entries, the first the server's executor


def request_paths(q: Request, sizes: Dict[str, List[Tuple[int, int]]],
                  max_passes: Optional[Dict[str, int]] = None) -> int:
    """Camera paths request q still has to render: its view's pixels x its
    remaining passes (passes 0: its scene's max_passes)."""
    w, h = sizes[q.scene][q.camera]
    return w * h * (total_passes(q, max_passes) - q.next_pass)


def total_passes(q: Request, max_passes: Optional[Dict[str, int]] = None) -> int:
    return q.passes or (max_passes or {}).get(q.scene, 1)


def path_weight(q: Request, layers: Optional[Dict[str, List[float]]] = None) -> float:
    """The cost of one camera path of q's view relative to a path that
    ends at its first surface: the view's surfel layers per path (each a
    walk step and a photon lookup), 1 when not measured."""
    if not layers or q.scene not in layers or q.camera >= len(layers[q.scene]):
        return 1.0
    return max(1.0, float(layers[q.scene][q.camera]))


def plan_round(queue: List[Request], sizes: Dict[str, List[Tuple[int, int]]], max_views: int,
               max_pixels: int, max_paths: Optional[int] = None,
               max_passes: Optional[Dict[str, int]] = None,
               max_scenes: int = MAX_ROUND_SCENES, policy: str = "arrival",
               now: float = 0.0, starve_s: float = 2.0,
               slices: bool = False,
               layers: Optional[Dict[str, List[float]]] = None,
               slice_gradients: bool = False) -> Tuple[List[Request], List[Request]]:
    """The requests of the next round, at most max_views views, max_pixels
    camera pixels, max_scenes distinct scenes and (when given) max_paths
    camera paths (request_paths); returns (taken, left), left in arrival
    order, and sets each taken request's round_passes (the passes it renders
    in the round, 0: all that remain).  policy "arrival": the queue's head
    in arrival order, up to the first request that does not fit.  policy
    "light_first": requests that have waited longer than starve_s first (in
    arrival order), then the others by their work (paths times the view's
    surfel layers per path from `layers`, per scene and camera, 1 when not
    given; a gradient request's counted twice), skipping those that do not
    fit, so that light requests are not held behind heavy ones and a heavy
    one waits at most about starve_s plus a round; the round's work is then
    also capped at 8 times its first request's (2^20 paths at least), so
    that requests of very different costs do not share a round.  With
    slices (and a path cap) a forward request over the cap that comes first
    renders as many of its passes as the cap holds, one at least, in a round
    of its own, and goes back to the queue for the rest: a heavy request
    advances in slices between which newly arrived requests get rounds; a
    gradient request too with slice_gradients (its loss and adjoint then
    run in the round of its last forward pass).  The first request
    considered always goes."""
    def work(q):
        return request_paths(q, sizes, max_passes) * path_weight(q, layers) * (2 if q.kind == "gradient" else 1)

    if policy == "arrival":
        order = list(queue)
    elif policy == "light_first":
        old = [q for q in queue if now - q.t_submit > starve_s]
        order = old + sorted((q for q in queue if not now - q.t_submit > starve_s), key=work)
    else:
        raise ValueError("policy must be 'arrival' or 'light_first'")
    taken, pix, paths, cost, scenes = [], 0, 0, 0.0, set()
    cap, cost_cap = max_paths, None
    for q in order:
        w, h = sizes[q.scene][q.camera]
        n = request_paths(q, sizes, max_passes)
        pw = path_weight(q, layers)
        k = 0                                  # all remaining passes
        fits = not taken or ((cap is None or paths + n <= cap)
                             and (cost_cap is None or cost + n * pw <= cost_cap))
        if not taken and slices and (q.kind == "forward" or slice_gradients) and cap is not None and n > cap:
            k = max(1, cap // (w * h))         # a first request over the cap renders a slice
        if taken and (not fits or len(taken) + 1 > max_views or pix + w * h > max_pixels
                      or (q.scene not in scenes and len(scenes) >= max_scenes)):
            if policy == "arrival":
                break
            continue
        q.round_passes = k
        m = w * h * k if k else n
        if not taken and policy == "light_first":
            # a round of light requests stays light: at most 8 times the
            # work of its first request (2^20 paths at least), so that a
            # light request does not wait for a heavy one in its own round
            cost_cap = max(float(1 << 20), 8.0 * m * pw)
        taken.append(q)
        pix += w * h
        paths += m
        cost += m * pw
        scenes.add(q.scene)
    chosen = set(map(id, taken))
    return taken, [q for q in queue if id(q) not in chosen]


class Server:
    """Resident scenes served in rounds of batched wavefronts (see the
    module docs)."""

    GRADIENTS_PER_WAVEFRONT = 8

    def __init__(self, hbm_budget: int, max_views: int = 64, max_pixels: int = 1 << 24,
                 settings: Optional[dict] = None, device: Optional[int] = None,
                 max_paths: Optional[int] = None, policy: str = "arrival", starve_s: float = 5.0,
                 slices: bool = True):
        import torch

        self.budget = int(hbm_budget)
        self.max_views = int(max_views)
        self.max_pixels = int(max_pixels)
        self.max_paths = None if max_paths is None else int(max_paths)
        if policy not in ("arrival", "light_first"):
            raise ValueError("policy must be 'arrival' or 'light_first'")
        self.policy, self.starve_s = policy, float(starve_s)
        self.slices = bool(slices) and self.max_paths is not None
        self.device = torch.device(f"cuda:{device if device is not None else torch.cuda.current_device()}")
        self.scenes: Dict[str, _Scene] = {}
        self.done: List[Request] = []
        self.rounds: List[int] = []           # views per round
        self._queue: List[Request] = []
        self._cv = threading.Condition()
        self._lock = threading.Lock()
        self._gpu = threading.Lock()          # the executor's buffers: one user at a time
        self._pin = None                      # pinned staging of the results
        self._stop = False
        # the executor: a tiny scene whose renderer lends the wavefront
        # buffers and the adjoint settings (rng mode, null weighting,
        # gradient groups, batch sizes) of every round
        # (gather estimator: the round's path vertices are kept within 16 GB
        # unless the settings say otherwise, the chunks past it replayed)
        st = {"gather_passes": 64, "adjoint_passes": 64, "adjoint_bounces": 8, "vertex_store_bytes": 16 << 30}
        st.update(settings or {})
        st.update(camera_seeds="camera", photons=1000, forward_passes=1)
        self._exec_settings = st
        self._gather = st.get("estimator", "reference") in ("gather", 1)
        # the gradient groups the adjoint writes (the others stay zero and
        # are not copied back)
        self._grad_keys = tuple(POINT_FIELDS) if st.get("gradients") in ("all", 1) else ("opacity",)
        self._exec = Renderer.from_scene(make_box_scene(8, cameras=1, resolution=8), st)
        # with the gather estimator, a second executor renders the forward-only
        # requests without keeping path vertices
        self._exec_plain = Renderer.from_scene(make_box_scene(8, cameras=1, resolution=8),
                                               dict(st, estimator="reference")) if self._gather else None
        self._thread = threading.Thread(target=self._run, name="pale-serve", daemon=True)
        self._thread.start()

    # ------------------------------------------------------------ scenes
    @property
    def admitted_bytes(self) -> int:
        return sum(s.footprint for s in self.scenes.values())

    def add_scene(self, name: str, scene: SceneArrays, settings: Optional[dict] = None) -> int:
        """Makes `scene` resident if it fits the budget (its photon map is
        traced now); returns the bytes it holds.  settings' gather/adjoint
        passes and adjoint bounces are the most a request may ask for."""
        if name in self.scenes:
            raise ValueError(f"scene '{name}' is already resident")
        import torch

        st = dict(settings or {})
        st["camera_seeds"] = "camera"
        torch.cuda.synchronize(self.device)
        before = _device_used()
        r = Renderer.from_scene(scene, st)
        try:
            self._photon_map(r)
            torch.cuda.synchronize(self.device)
            footprint = max(0, _device_used() - before)
        except Exception:
            r.close()
            raise
        if self.admitted_bytes + footprint > self.budget:
            r.close()
            raise AdmissionError(f"scene '{name}' needs {footprint / 2**30:.2f} GiB; "
                                 f"{(self.budget - self.admitted_bytes) / 2**30:.2f} GiB of the budget left")
        try:
            layers = self._layers(r)
        except Exception:
            r.close()
            raise
        with self._cv:
            self.scenes[name] = _Scene(name, r, footprint, min(int(r._settings.gather_passes),
                                                               int(r._settings.adjoint_passes)),
                                       int(r._settings.adjoint_bounces), layers)
        return footprint

    def _layers(self, r: Renderer) -> List[float]:
        """Surfel layers per camera path of each of r's cameras (gather
        segments per path of one pass of the camera alone, on the executor
        that keeps no path vertices): the planner's cost of a path of that
        view.  A view into a dense cloud costs two orders of magnitude more
        per path than one of a wall."""
        from .device import ViewBatch

        ex = self._exec_plain if self._exec_plain is not None else self._exec
        out = []
        with self._gpu:
            for c, (w, h) in enumerate(r._sizes):
                ViewBatch([ex, r], [(1, c, 1, 0)], device=self.device).forward_loss(None, trace_photons=False)
                out.append(ex.stats()["gather_segments"] / float(max(1, w * h)))
        return out

    def _photon_map(self, r: Renderer):
        """Traces the scene's photon map, which then stays resident."""
        import ctypes as C

        import torch

        from .pale import _check

        stream = C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        _check(r._lib, r._h, r._lib.pale_trace_photon_map(r._h, stream), "trace_photon_map")

    def remove_scene(self, name: str):
        with self._cv:
            sc = self.scenes.pop(name)
        sc.renderer.close()

    # ---------------------------------------------------------- requests
    def submit(self, req: Request) -> Request:
        sc = self.scenes.get(req.scene)
        if sc is None:
            raise KeyError(f"scene '{req.scene}' is not resident")
        if req.kind not in ("forward", "gradient"):
            raise ValueError("kind must be 'forward' or 'gradient'")
        if not 0 <= req.camera < len(sc.renderer._names):
            raise IndexError("camera index out of range")
        if req.kind == "gradient" and req.target is None:
            raise ValueError("a gradient request needs a target image")
        if not 0 <= req.passes <= sc.max_passes:
            raise ValueError(f"passes must be 0 .. {sc.max_passes}")
        if not 0 <= req.depth <= sc.max_depth:
            raise ValueError(f"depth must be 0 .. {sc.max_depth}")
        req.t_submit = time.perf_counter()
        with self._cv:
            self._queue.append(req)
            self._cv.notify()
        with self._lock:
            self.done.append(req)
        return req

    # ------------------------------------------------------------ rounds
    def _host(self, t) -> np.ndarray:
        """A host copy of device tensor `t` through a pinned staging buffer
        (device-to-host copies from pinned memory run at several times the
        rate of pageable ones)."""
        import torch

        n = t.numel()
        if self._pin is None or self._pin.numel() < n:
            self._pin = torch.empty(max(n, 1 << 20), dtype=torch.float32, pin_memory=True)
        buf = self._pin[:n].view(t.shape)
        buf.copy_(t)
        return buf.numpy().copy()

    def _host_grads(self, g) -> Dict[str, np.ndarray]:
        """Host copies of the computed gradient groups of `g`, staged
        through the pinned buffer with one synchronisation."""
        import torch

        keys = [k for k in self._grad_keys if k in g]
        n = sum(g[k].numel() for k in keys)
        if self._pin is None or self._pin.numel() < n:
            self._pin = torch.empty(max(n, 1 << 20), dtype=torch.float32, pin_memory=True)
        views, off = [], 0
        for k in keys:
            t = g[k]
            buf = self._pin[off:off + t.numel()].view(t.shape)
            buf.copy_(t, non_blocking=True)
            views.append((k, buf))
            off += t.numel()
        torch.cuda.current_stream(self.device).synchronize()
        return {k: buf.numpy().copy() for k, buf in views}

    def _run(self):
        import torch

        torch.cuda.set_device(self.device)
        while True:
            with self._cv:
                while not self._queue and not self._stop:
                    self._cv.wait()
                if self._stop and not self._queue:
                    return
                sizes = {n: s.renderer._sizes for n, s in self.scenes.items()}
                spp = {n: s.max_passes for n, s in self.scenes.items()}
                layers = {n: s.layers for n, s in self.scenes.items()}
                taken, self._queue = plan_round(self._queue, sizes, self.max_views, self.max_pixels,
                                                self.max_paths, spp, policy=self.policy,
                                                now=time.perf_counter(), starve_s=self.starve_s,
                                                slices=self.slices, layers=layers,
                                                slice_gradients=not self._gather)
            try:
                with self._gpu:
                    self._round(taken)
            except Exception as e:  # reported per request
                for q in taken:
                    if not q.done.is_set():
                        q.error = str(e)
            now = time.perf_counter()
            again = []
            for q in taken:
                if q.done.is_set():
                    continue
                if q.error is None and q.partial is not None:
                    again.append(q)          # a slice done, passes left: back to the queue
                    continue
                q.t_done = now
                q.done.set()
            if again:
                with self._cv:
                    self._queue = sorted(self._queue + again, key=lambda r: r.t_submit)

    def _round(self, reqs: List[Request]):
        import torch

        from .device import ViewBatch

        n_round = len(self.rounds)
        self.rounds.append(len(reqs))
        names = sorted({q.scene for q in reqs})
        entry = {n: k + 1 for k, n in enumerate(names)}     # entry 0: the executor
        scene_renderers = [self.scenes[n].renderer for n in names]

        def passes(q):
            return q.passes or self.scenes[q.scene].max_passes

        def forward(idx, executor):
            """One forward wavefront over requests idx: images to the host,
            the L2 loss and dL/dI of its gradient requests (compute_l2_loss
            / compute_l2_grad, python/losses.py:10-45, on the LDR image).  A
            forward request with a slice renders those passes, its running
            sums carried between rounds; it is finished (and its image read)
            in the round of its last pass."""
            views, ranges = [], []
            for i in idx:
                q = reqs[i]
                P = passes(q)
                k = q.round_passes or P - q.next_pass
                rng = (q.next_pass, k) if (q.next_pass or k < P) else (0, 0)
                ranges.append(rng)
                views.append((entry[q.scene], q.camera, P, q.depth) + rng)
            vb = ViewBatch([executor] + scene_renderers, views, device=self.device)
            offs = np.cumsum([0] + [w * h for w, h in vb.sizes])
            partial = None
            if vb.sliced:
                partial = torch.zeros(max(1, int(offs[-1])), 4, dtype=torch.float32, device=self.device)
                for k, i in enumerate(idx):
                    if ranges[k][0] > 0:
                        partial[offs[k]:offs[k + 1]].copy_(reqs[i].partial)
            vb.forward_loss(None, trace_photons=False, partial=partial)   # the resident photon maps
            finished = []
            for k, i in enumerate(idx):
                q = reqs[i]
                first, count = ranges[k]
                q.slices += 1
                if count and first + count < passes(q):
                    q.next_pass = first + count
                    q.partial = partial[offs[k]:offs[k + 1]].clone()
                else:
                    q.next_pass, q.partial = passes(q), None
                    finished.append(k)
            dldi = {}
            done_now = set(finished)
            for k, i in enumerate(idx):
                q = reqs[i]
                if q.kind != "gradient" or k not in done_now:
                    continue   # (a sliced gradient request's loss waits for its last slice)
                t = torch.from_numpy(np.ascontiguousarray(q.target, np.float32).reshape(-1, 3)).to(self.device)
                d = torch.zeros(int(offs[k + 1] - offs[k]), 4, dtype=torch.float32, device=self.device)
                torch.sub(vb.ldr[offs[k]:offs[k + 1], :3], t, out=d[:, :3])
                q.loss = float((0.5 * (d[:, :3].double() ** 2).mean()).item())
                d[:, :3].div_(float(3 * (offs[k + 1] - offs[k])))
                dldi[i] = d
            ldr = self._host(vb.ldr)
            for k in finished:
                q = reqs[idx[k]]
                w, h = vb.sizes[k]
                q.image = ldr[offs[k]:offs[k + 1]].reshape(h, w, 4).copy()
                q.batch_views = len(reqs)
                q.round = n_round
                if q.kind != "gradient":
                    q.t_done = time.perf_counter()
                    q.done.set()
            return vb, offs, dldi

        def finish(idx, host):
            now = time.perf_counter()
            for k, i in enumerate(idx):
                reqs[i].grads = host[k]
                reqs[i].t_done = now
                reqs[i].done.set()

        grad_idx = [i for i, q in enumerate(reqs) if q.kind == "gradient"]
        plain_idx = [i for i, q in enumerate(reqs) if q.kind != "gradient"]
        if self._gather:
            # forward-only requests on the reference executor (no path
            # vertices kept); the gradient requests' own forward on the
            # gather executor, then one sweep over its vertices, each view
            # into arrays of its own
            if plain_idx:
                forward(plain_idx, self._exec_plain)
            if grad_idx:
                vb, offs, dldi = forward(grad_idx, self._exec)
                dl = torch.cat([dldi[i] for i in grad_idx]).contiguous()
                gl = vb.view_gradients(list(range(len(grad_idx))), dl)
                finish(grad_idx, [self._host_grads(g) for g in gl])
            return
        vb, offs, dldi = forward(list(range(len(reqs))), self._exec)
        grad_idx = [i for i in grad_idx if i in dldi]   # those whose image is finished
        per = self.GRADIENTS_PER_WAVEFRONT - 1     # entry 0 is the executor
        for c0 in range(0, len(grad_idx), per):
            chunk = grad_idx[c0:c0 + per]
            # one scene entry per request, so each request keeps its own gradients
            rs = [self._exec] + [self.scenes[reqs[i].scene].renderer for i in chunk]
            gviews = [(k + 1, reqs[i].camera, passes(reqs[i]), reqs[i].depth) for k, i in enumerate(chunk)]
            gb = ViewBatch(rs, gviews, device=self.device)
            dl = torch.cat([dldi[i] for i in chunk]).contiguous()
            grads = gb.backward(dl)
            finish(chunk, [self._host_grads(grads[e + 1]) for e in range(len(chunk))])

    # ----------------------------------------------------------- reports
    def latency(self, kind: Optional[str] = None) -> Dict[str, float]:
        """p50 / p99 / mean latency (ms) of the finished requests."""
        with self._lock:
            lat = [q.latency_ms for q in self.done if q.done.is_set() and (kind is None or q.kind == kind)]
        if not lat:
            return {"n": 0}
        a = np.asarray(lat)
        return {"n": int(a.size), "p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)),
                "mean": float(a.mean())}

    def serve_one(self, req: Request) -> Request:
        """The plain path: `req` rendered alone, right now, on the calling
        thread, waiting for any round in flight (no batching: the
        one-request-at-a-time baseline, and the check that a request's
        result does not depend on its round)."""
        req.t_submit = time.perf_counter()
        with self._gpu:
            saved = list(self.rounds)
            try:
                self._round([req])
            finally:
                self.rounds = saved
        if not req.done.is_set():
            req.t_done = time.perf_counter()
            req.done.set()
        return req

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify()
        self._thread.join()
        for name in list(self.scenes):
            self.remove_scene(name)
        self._exec.close()
        if self._exec_plain is not None:
            self._exec_plain.close()
