"""``pale.Renderer`` on the B200 renderer.

This module mirrors the pybind11 surface of Pale (Pale/pale_bindings.cpp:
1613-1650) -- method names, argument names and defaults, dict keys, array
shapes and error types -- so Pale's optimisation loop (python/training.py,
python/render_hooks.py) and its finite-difference scripts run unchanged with
``import differentiablepointrendering_b200.pale as pale``.

Every call goes through the C-ABI of ``libpale_b200.so``; there is no CPU
path.  Arrays returned are fresh host copies; parameters and gradients are
in BVH order, as in the reference.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from .scene import (POINT_FIELDS, POINT_WIDTH, SceneArrays, as_points, load_mitsuba_scene, load_surfel_ply,
                    resolve_point_cloud)


def _check(lib, h, rc: int, what: str):
    if rc != 0:
        msg = lib.pale_last_error(h)
        msg = msg.decode(errors="replace") if msg else ""
        raise RuntimeError(f"{what} failed ({rc}): {msg}")


def _split_rgba(buf: np.ndarray, sizes) -> list:
    """(H, W, 4) views of consecutive cameras' pixels in one packed float32
    buffer; `sizes` holds (W, H) per camera."""
    out, off = [], 0
    for w, h in sizes:
        n = w * h * 4
        out.append(buf[off:off + n].reshape(h, w, 4))
        off += n
    return out


def _packed_parent(rgbs):
    """The packed float32 RGBA buffer whose consecutive (H, W, 4) images
    the (H, W, 3) arrays `rgbs` are, in order, the RGB views of (as
    render_forward_loss returns dL/dI), or None."""
    if not rgbs:
        return None

    def root(a):
        while isinstance(a.base, np.ndarray):
            a = a.base
        return a

    r = root(rgbs[0])
    if r.dtype != np.float32 or not r.flags.c_contiguous:
        return None
    p0, off = r.__array_interface__["data"][0], 0
    for a in rgbs:
        h, w, _ = a.shape
        if (a.dtype != np.float32 or a.strides != (16 * w, 16, 4) or root(a) is not r
                or a.__array_interface__["data"][0] != p0 + 16 * off):
            return None
        off += h * w
    if r.size < 4 * off:
        return None
    return r.reshape(-1)[:4 * off]


def _pack_rgba(rgbs) -> tuple:
    """One packed float32 buffer of (H, W, 3) images with alpha 1 (the
    layout the C-ABI reads), and its (H, W, 4) view per image; a 4-float
    zero buffer and no views when there are no images."""
    n = sum(a.shape[0] * a.shape[1] for a in rgbs) * 4
    if n == 0:
        return np.zeros(4, np.float32), []
    sizes = [(a.shape[1], a.shape[0]) for a in rgbs]
    buf = _packed_parent(rgbs)
    if buf is not None:
        # the RGB views of one packed buffer: passed in place (its alpha,
        # which no view shows, set to 1)
        views = _split_rgba(buf, sizes)
        for v in views:
            v[..., 3] = 1.0
        return buf, views
    buf = np.empty(n, np.float32)
    views = _split_rgba(buf, sizes)
    for v, a in zip(views, rgbs):
        v[..., :3] = a
        v[..., 3] = 1.0
    return buf, views


class Renderer:
    """Adjoint photon-mapping renderer for beta surfels on one B200.

    Renderer(assetRootDir, sceneXml="cbox_custom.xml",
             pointCloudFile="initial.ply", settings={})
    """

    def __init__(self, assetRootDir: str, sceneXml: str = "cbox_custom.xml",
                 pointCloudFile: str = "initial.ply", settings: Optional[dict] = None,
                 *, scene: Optional[SceneArrays] = None):
        self._lib = N.load_library()
        self._h = C.c_void_p()
        if scene is None:
            root = os.path.abspath(assetRootDir)
            pts = load_surfel_ply(resolve_point_cloud(root, pointCloudFile))
            scene = load_mitsuba_scene(root, sceneXml, pts)
        self._scene = scene
        self._settings = N.settings_from_dict(settings)
        self._asset_host = {k: v.copy() for k, v in as_points(scene.points).items()}
        self._asset_stale = False   # the device asset is newer (optimizer_step)
        desc = N.SceneDescHolder(scene)
        rc = self._lib.pale_create(C.byref(desc.struct), C.byref(self._settings), C.byref(self._h))
        if rc != 0:
            msg = self._lib.pale_last_error(None)
            raise RuntimeError(f"pale_create failed ({rc}): {msg.decode(errors='replace') if msg else ''}")
        self._names = list(scene.camera_names)
        self._sizes = [(int(w), int(h)) for w, h in scene.camera_size]
        self._adjoint = [bool(a) for a in scene.camera_adjoint]

    @classmethod
    def from_scene(cls, scene: SceneArrays, settings: Optional[dict] = None) -> "Renderer":
        """Renderer over in-memory scene arrays (no files)."""
        return cls("", settings=settings, scene=scene)

    # ------------------------------------------------------------ basics
    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.pale_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_camera_names(self) -> List[str]:
        return list(self._names)

    @property
    def num_points(self) -> int:
        n = C.c_uint32()
        _check(self._lib, self._h, self._lib.pale_point_count(self._h, C.byref(n)), "pale_point_count")
        return int(n.value)

    @property
    def settings(self) -> N.PaleSettings:
        return self._settings

    # ----------------------------------------------------------- forward
    def render_forward(self, camera_name: str = "") -> Dict[str, np.ndarray]:
        """{cam: LDR (H,W,4), cam+'_raw': HDR (H,W,4)} float32
        (render_forward, pale_bindings.cpp:180-277)."""
        return self._render(camera_name, self._lib.pale_render_forward, "render_forward")

    def render_gather(self, camera_name: str = "") -> Dict[str, np.ndarray]:
        """render_forward without retracing the photons: the camera gather
        from the current photon map (the last forward's or loaded photons),
        with the last forward's camera seeds."""
        return self._render(camera_name, self._lib.pale_render_gather, "render_gather")

    def _render(self, camera_name, fn, what) -> Dict[str, np.ndarray]:
        idx = [i for i, n in enumerate(self._names) if (not camera_name or n == camera_name)]
        pix = sum(self._sizes[i][0] * self._sizes[i][1] for i in idx)
        ldr = np.empty(max(1, pix) * 4, np.float32)
        raw = np.empty(max(1, pix) * 4, np.float32)
        cams = N.cams_array(idx)
        rc = fn(self._h, len(idx), cams.ctypes.data_as(N.u32p), ldr.ctypes.data_as(N.f32p), raw.ctypes.data_as(N.f32p))
        _check(self._lib, self._h, rc, what)
        out, off = {}, 0
        for i in idx:
            w, h = self._sizes[i]
            n = w * h * 4
            out[self._names[i]] = ldr[off:off + n].reshape(h, w, 4).copy()
            out[self._names[i] + "_raw"] = raw[off:off + n].reshape(h, w, 4).copy()
            off += n
        return out

    def render_forward_loss(self, targets: Dict[str, np.ndarray]):
        """render_forward of the cameras named in `targets` ({cam: (H,W,3)
        or (H,W,4) float32, alpha ignored}) with the training loop's L2
        loss computed by the post-process (compute_l2_grad /
        compute_l2_loss, python/losses.py:10-45): returns (images as
        render_forward, {cam: dL/dI (H,W,3) float32}, {cam: loss})."""
        idx = [i for i, n in enumerate(self._names) if n in targets]
        if len(idx) != len(targets):
            raise RuntimeError(f"unknown camera in targets: {sorted(set(targets) - set(self._names))}")
        chans = {np.asarray(targets[self._names[i]]).shape[-1] for i in idx}
        if len(chans) > 1 or not chans <= {3, 4}:
            raise RuntimeError("target images must all be (H,W,3) or all (H,W,4)")
        ch = chans.pop() if chans else 3
        parts = []
        for i in idx:
            w, h = self._sizes[i]
            t = np.asarray(targets[self._names[i]], np.float32)
            if t.shape != (h, w, ch):
                raise RuntimeError(f"target for {self._names[i]} must have shape {(h, w, ch)}, got {t.shape}")
            parts.append(t.reshape(-1))
        tgt = np.ascontiguousarray(np.concatenate(parts) if parts else np.zeros(ch, np.float32))
        pix = sum(self._sizes[i][0] * self._sizes[i][1] for i in idx)
        ldr = np.empty(max(1, pix) * 4, np.float32)
        raw = np.empty(max(1, pix) * 4, np.float32)
        dldi = np.empty(max(1, pix) * 4, np.float32)
        loss = np.zeros(max(1, len(idx)), np.float64)
        cams = N.cams_array(idx)
        rc = self._lib.pale_render_forward_loss(self._h, len(idx), cams.ctypes.data_as(N.u32p),
                                                tgt.ctypes.data_as(N.f32p), ch, ldr.ctypes.data_as(N.f32p),
                                                raw.ctypes.data_as(N.f32p), dldi.ctypes.data_as(N.f32p),
                                                loss.ctypes.data_as(C.POINTER(C.c_double)))
        _check(self._lib, self._h, rc, "render_forward_loss")
        # the images are views of this call's buffers (no further copy)
        sizes = [self._sizes[i] for i in idx]
        images, grads, losses = {}, {}, {}
        for k, (i, l4, r4, d4) in enumerate(zip(idx, _split_rgba(ldr, sizes), _split_rgba(raw, sizes),
                                                _split_rgba(dldi, sizes))):
            name = self._names[i]
            images[name] = l4
            images[name + "_raw"] = r4
            grads[name] = d4[..., :3]          # a view: render_backward takes it in place
            losses[name] = float(loss[k])
        return images, grads, losses

    # ---------------------------------------------------------- backward
    def render_backward(self, targetRgb32f: Dict[str, np.ndarray]) -> Tuple[dict, dict]:
        """Adjoint pass with dL/dI images {cam: (H,W,3) float32}; returns
        (gradients, {"adjoint_source": {...}[, "debug": {...}]})
        (render_backward, pale_bindings.cpp:279-731)."""
        idx, imgs = [], []
        for i, name in enumerate(self._names):
            if not self._adjoint[i] or name not in targetRgb32f:
                continue
            arr = np.asarray(targetRgb32f[name])
            if arr.ndim != 3 or arr.shape[2] != 3:
                raise RuntimeError(f"render_backward: target image for camera '{name}' must be HxWx3 float32")
            if arr.dtype.itemsize != 4:
                raise RuntimeError(f"render_backward: target image for camera '{name}' must have dtype float32")
            h, w = arr.shape[0], arr.shape[1]
            sw, sh = self._sizes[i]
            if w != sw or h != sh:
                raise RuntimeError(f"render_backward: resolution mismatch for camera '{name}': target image is "
                                   f"{w}x{h}, but sensor is {sw}x{sh}")
            idx.append(i)
            imgs.append(arr.view(np.float32).reshape(h, w, 3))
        # one packed RGBA buffer; the returned adjoint sources are its views
        dldi, imgs = _pack_rgba(imgs)
        n = self.num_points
        grads = N.PointsHolder(n=n)
        pix = sum(im.size for im in imgs)
        dbg = np.zeros(max(4, pix), np.float32) if self._settings.debug_images else None
        cams = N.cams_array(idx)
        rc = self._lib.pale_render_backward(self._h, len(idx), cams.ctypes.data_as(N.u32p),
                                            dldi.ctypes.data_as(N.f32p), C.byref(grads.struct),
                                            dbg.ctypes.data_as(N.f32p) if dbg is not None else None)
        _check(self._lib, self._h, rc, "render_backward")
        g = {k: grads.arrays[k] for k in POINT_FIELDS}   # this call's own arrays
        images = {"adjoint_source": {self._names[i]: im for i, im in zip(idx, imgs)}}
        if self._settings.debug_images:
            dbg_out, off = {}, 0
            for i, im in zip(idx, imgs):
                k = im.size
                zero = np.zeros_like(im)
                op = dbg[off:off + k].reshape(im.shape).copy()
                dbg_out[self._names[i]] = {"position_x": zero, "position_y": zero.copy(),
                                           "position_z": zero.copy(), "rotation": zero.copy(),
                                           "scale": zero.copy(), "albedo": zero.copy(), "opacity": op,
                                           "beta": zero.copy()}
                off += k
            images["debug"] = dbg_out
        return g, images

    # -------------------------------------------------------- parameters
    def get_point_parameters(self) -> Dict[str, np.ndarray]:
        """Surfel parameters in BVH order (pale_bindings.cpp:733-850)."""
        out = N.PointsHolder(n=self.num_points)
        _check(self._lib, self._h, self._lib.pale_get_points(self._h, C.byref(out.struct)), "get_point_parameters")
        return {k: out.arrays[k].copy() for k in POINT_FIELDS}

    def get_point_order(self) -> np.ndarray:
        """order[bvh_index] = asset index of the last BVH build."""
        o = np.zeros(max(1, self.num_points), np.uint32)
        _check(self._lib, self._h, self._lib.pale_get_order(self._h, o.ctypes.data_as(N.u32p)), "get_order")
        return o[: self.num_points].copy()

    def apply_point_optimization(self, parameters: Dict[str, np.ndarray]):
        """Writes BVH-ordered parameters without a BVH rebuild and mirrors
        them into the asset (pale_bindings.cpp:853-1056)."""
        if "position" not in parameters:
            return
        pos = np.asarray(parameters["position"])
        if pos.ndim != 2 or pos.shape[1] != 3:
            raise RuntimeError("Expected 'position' to have shape (N,3)")
        n_in, n = pos.shape[0], self.num_points
        if n_in == 0:
            return
        if n_in != n:
            raise RuntimeError("apply_point_optimization expects consistent point count; "
                               "use densification API for adding/removing points.")
        cur = self.get_point_parameters()
        for key, width in (("position", 3), ("tangent_u", 3), ("tangent_v", 3), ("scale", 2), ("albedo", 3),
                           ("opacity", 1), ("beta", 1)):
            if key not in parameters:
                raise RuntimeError("New points dictionary does not contain key: " + key)
            a = np.asarray(parameters[key])
            shape_ok = (a.ndim == 2 and a.shape == (n, width)) if width > 1 else (a.ndim == 1 and a.shape[0] == n)
            if not shape_ok:
                raise RuntimeError(f"Expected '{key}' to have shape (N,{width})" if width > 1
                                   else f"Expected '{key}' to have shape (N,)")
            if a.dtype.itemsize != 4:
                raise RuntimeError(f"Expected '{key}' to be float32")
            cur[key] = np.ascontiguousarray(a).view(np.float32).reshape(cur[key].shape).copy()
        hold = N.PointsHolder(cur)
        _check(self._lib, self._h, self._lib.pale_apply_points(self._h, C.byref(hold.struct)),
               "apply_point_optimization")
        for key in ("position", "tangent_u", "tangent_v", "scale", "albedo", "opacity", "beta"):
            self._asset[key] = cur[key].copy()

    def rebuild_bvh(self):
        """Rebuilds the surfel LBVH from the asset (pale_bindings.cpp:1058-1079)."""
        if self._asset_stale:       # the device holds the newest asset
            _check(self._lib, self._h, self._lib.pale_rebuild(self._h, None), "rebuild_bvh")
            return
        hold = N.PointsHolder(self._asset)
        _check(self._lib, self._h, self._lib.pale_rebuild(self._h, C.byref(hold.struct)), "rebuild_bvh")

    @property
    def _asset(self) -> Dict[str, np.ndarray]:
        """Host copy of the asset, fetched from the device after optimizer steps."""
        if self._asset_stale:
            out = N.PointsHolder(n=self.num_points)
            _check(self._lib, self._h, self._lib.pale_get_asset(self._h, C.byref(out.struct)), "get_asset")
            self._asset_host = {k: out.arrays[k].copy() for k in POINT_FIELDS}
            self._asset_stale = False
        return self._asset_host

    @_asset.setter
    def _asset(self, value: Dict[str, np.ndarray]):
        self._asset_host = value
        self._asset_stale = False

    # ------------------------------------------------------- training step
    def optimizer_step(self, config: Optional[dict] = None, opacity_reset: Optional[float] = None, stream=None,
                       grads: Optional[Dict[str, object]] = None):
        """One optimizer step of the training loop on the device
        (training.py:685-743): the gradients of the last render_backward go
        through Adam / SGD / MaskedAdam with per-group learning rates
        (OptimizationConfig keys, optimizers.py:11-66), opacities are set to
        `opacity_reset` if given, the parameters are projected onto their
        constraints (verify_parameters_inplane) and written back without a
        BVH rebuild (apply_point_optimization).  Optimizer state stays on
        the device and starts over after each BVH rebuild, as the reference
        creates a new optimizer then.  Runs on `stream` (a torch.cuda.Stream
        or a raw handle; None = the default stream) without waiting.
        `grads` replaces the adjoint's gradients by CUDA tensors (float32,
        contiguous, BVH order) of the seven fields."""
        opt = N.optimizer_from_config(config, opacity_reset)
        if stream is None or isinstance(stream, C.c_void_p):
            s = stream
        else:
            s = C.c_void_p(int(getattr(stream, "cuda_stream", stream)))
        g = None
        if grads is not None:
            g = N.PalePoints()
            g.count = self.num_points
            for k in POINT_FIELDS[:7]:
                t = grads[k]
                if not (t.is_cuda and t.is_contiguous() and str(t.dtype) == "torch.float32"):
                    raise ValueError(f"optimizer_step: gradient '{k}' must be a contiguous float32 CUDA tensor")
                if t.numel() != self.num_points * POINT_WIDTH[k]:
                    raise ValueError(f"optimizer_step: gradient '{k}' has {t.numel()} entries")
                setattr(g, k, C.cast(C.c_void_p(t.data_ptr()), N.f32p))
            g = C.byref(g)
        _check(self._lib, self._h, self._lib.pale_optimizer_step(self._h, C.byref(opt), g, s), "optimizer_step")
        self._asset_stale = True

    # ------------------------------------------------------ density control
    def prune_by_opacity(self, min_opacity: float, use_quantile: bool = True, max_fraction_to_prune: float = 0.3,
                         min_points_to_keep: int = 1) -> np.ndarray:
        """compute_prune_indices_by_opacity (density_control.py:199-263) on
        the device asset, then remove_points + rebuild_bvh, in one call.
        Returns the removed asset indices in increasing order (what
        np.unique of the reference's indices gives)."""
        n = self.num_points
        out = np.zeros(max(1, n), np.int64)
        cnt = C.c_uint32()
        _check(self._lib, self._h,
               self._lib.pale_prune_by_opacity(self._h, float(min_opacity), 1 if use_quantile else 0,
                                               float(max_fraction_to_prune), int(min_points_to_keep), C.byref(cnt),
                                               out.ctypes.data_as(C.POINTER(C.c_int64))), "prune_by_opacity")
        if cnt.value:
            self._asset_stale = True
        return out[:cnt.value].copy()

    def densify_long_axis_split(self, importance=None, max_new_points: Optional[int] = None,
                                split_distance: float = 0.6, minor_axis_shrink: float = 0.85,
                                opacity_reduction: float = 0.6, min_long_axis_scale: float = 0.0,
                                grad_threshold: float = 0.0) -> np.ndarray:
        """densify_points_long_axis_split (density_control.py:6-196) on the
        device asset, then remove_points(parents) + add_points(children) +
        rebuild_bvh.  `importance` (one score per surfel, asset order) may be
        a CUDA tensor or a host array.  Returns the parent indices."""
        n = self.num_points
        keep = None
        ptr = None
        if importance is not None:
            if hasattr(importance, "is_cuda") and importance.is_cuda:
                keep = importance.detach().float().contiguous().reshape(-1)
            else:
                import torch
                keep = torch.from_numpy(np.ascontiguousarray(np.asarray(importance, np.float32).reshape(-1))).cuda()
            if keep.numel() != n:
                raise ValueError(f"importance needs {n} scores, got {keep.numel()}")
            ptr = C.c_void_p(keep.data_ptr())
        budget = -1 if max_new_points is None else int(max_new_points)
        if max_new_points is not None and int(max_new_points) // 2 <= 0:
            return np.zeros(0, np.int64)
        out = np.zeros(max(1, n), np.int64)
        cnt = C.c_uint32()
        if keep is not None:
            import torch
            torch.cuda.synchronize()
        _check(self._lib, self._h,
               self._lib.pale_densify_long_axis_split(self._h, ptr, budget, float(split_distance),
                                                      float(minor_axis_shrink), float(opacity_reduction),
                                                      float(min_long_axis_scale), float(grad_threshold), C.byref(cnt),
                                                      out.ctypes.data_as(C.POINTER(C.c_int64))),
               "densify_long_axis_split")
        if cnt.value:
            self._asset_stale = True
        return out[:cnt.value].copy()

    def reset_optimizer(self):
        """Drops the device optimizer state (zero moments at the next step)."""
        _check(self._lib, self._h, self._lib.pale_optimizer_reset(self._h), "reset_optimizer")

    def remove_points(self, parameters: Dict[str, np.ndarray]):
        """Removes asset points by index, then rebuilds (:1081-1189)."""
        if "indices" not in parameters:
            raise RuntimeError("remove_points: expected key 'indices' (1D int32 / int64 array)")
        ind = np.asarray(parameters["indices"])
        if ind.ndim != 1:
            raise RuntimeError("remove_points: 'indices' must be a 1D array")
        if ind.shape[0] == 0:
            return
        if ind.dtype not in (np.int32, np.int64, np.uint32, np.uint64):
            raise RuntimeError("remove_points: 'indices' must have dtype int32 or int64")
        n = self._asset["position"].shape[0]
        if n == 0:
            return
        keep = np.ones(n, bool)
        for v in ind.tolist():
            if v < 0:
                raise IndexError("remove_points: negative index is not allowed")
            if v >= n:
                raise IndexError("remove_points: index out of range")
            keep[v] = False
        self._asset = {k: v[keep].copy() for k, v in self._asset.items()}
        self.rebuild_bvh()

    def add_points(self, parameters: Dict[str, dict]):
        """Appends points given as {"new": {...7 keys}}, then rebuilds
        (add_new_points, :1191-1395)."""
        if "new" not in parameters:
            return
        new = parameters["new"]
        for key in ("position", "tangent_u", "tangent_v", "scale", "albedo", "opacity", "beta"):
            if key not in new:
                raise RuntimeError(f"add_new_points: missing key 'new.{key}'")
        pos = np.asarray(new["position"])
        if pos.ndim != 2 or pos.shape[1] != 3:
            raise RuntimeError("add_new_points: 'new.position' must have shape (N,3)")
        if pos.dtype.itemsize != 4:
            raise RuntimeError("add_new_points: 'new.position' must be float32")
        m = pos.shape[0]
        if m == 0:
            return
        for key, width in (("tangent_u", 3), ("tangent_v", 3), ("scale", 2), ("albedo", 3)):
            a = np.asarray(new[key])
            if a.ndim != 2 or a.shape != (m, width):
                raise RuntimeError(f"add_new_points: 'new.{key}' must have shape (N,{width})")
            if a.dtype.itemsize != 4:
                raise RuntimeError(f"add_new_points: 'new.{key}' must be float32")
        for key in ("opacity", "beta"):
            a = np.asarray(new[key])
            if a.ndim != 1 or a.shape[0] != m:
                raise RuntimeError("add_new_points: 'new.opacity' must have shape (N,)")
            if a.dtype.itemsize != 4:
                raise RuntimeError("add_new_points: 'new.opacity' must be float32")
        add = as_points({k: np.ascontiguousarray(np.asarray(new[k])).view(np.float32) for k in
                         ("position", "tangent_u", "tangent_v", "scale", "albedo", "opacity", "beta")})
        add["shape"] = np.zeros(m, np.float32)
        self._asset = {k: np.concatenate([self._asset[k], add[k]]) for k in POINT_FIELDS}
        self.rebuild_bvh()

    def set_point_opacity(self, opacity: float, index: int):
        n = self._asset["opacity"].shape[0]
        if index < 0 or index >= n:
            raise RuntimeError("set_gaussian_opacity: index out of range")
        self._asset["opacity"][index] = np.float32(opacity)
        self.rebuild_bvh()

    def set_point_beta(self, beta: float, index: int):
        n = self._asset["opacity"].shape[0]
        if index < 0 or index >= n:
            raise RuntimeError("set_point_beta: index out of range")
        self._asset["beta"][index] = np.float32(beta)
        self.rebuild_bvh()

    def set_point_properties(self, translation3, rotation_quat4, scale3, albedo3, opacity: float, beta: float,
                             index: int = -1):
        """Perturbs asset points (pale_bindings.cpp:1485-1600).  With
        index < 0 the reference's loop advances by two, so every second
        point is perturbed; that behaviour is kept."""
        if len(translation3) != 3 or len(rotation_quat4) != 4 or len(scale3) != 3:
            raise RuntimeError("Expected translation(3), rotation_quat(4), scale(3)")
        t = np.asarray(translation3, np.float32)
        col = np.asarray(albedo3, np.float32)
        qx, qy, qz, qw = (np.float32(v) for v in rotation_quat4)
        sc = np.asarray(scale3[:2], np.float32)
        A = self._asset
        n = A["position"].shape[0]

        def rot(v):
            qv = np.array([qx, qy, qz], np.float32)
            uv = np.cross(qv, v).astype(np.float32)
            uuv = np.cross(qv, uv).astype(np.float32)
            return (v + ((uv * qw) + uuv) * np.float32(2)).astype(np.float32)

        if index < 0:
            for i in range(0, n, 2):
                A["position"][i] += t
                A["tangent_u"][i] = rot(A["tangent_u"][i])
                A["tangent_v"][i] = rot(A["tangent_v"][i])
                A["albedo"][i] += col
                A["opacity"][i] += np.float32(opacity)
                A["beta"][i] += np.float32(beta)
                A["scale"][i] *= sc
        else:
            if index > n - 1:
                raise RuntimeError("add_new_points: index out of range")
            A["position"][index] += t
            A["tangent_u"][index] = rot(A["tangent_u"][index])
            A["tangent_v"][index] = rot(A["tangent_v"][index])
            A["albedo"][index] = col
            A["opacity"][index] = np.float32(opacity)
            A["beta"][index] = np.float32(beta)
            A["scale"][index] = sc
        self.rebuild_bvh()

    # ------------------------------------------------------- diagnostics
    def stats(self) -> Dict[str, float]:
        st = N.PaleStats()
        _check(self._lib, self._h, self._lib.pale_get_stats(self._h, C.byref(st)), "get_stats")
        return st.as_dict()

    def trace_rays(self, origins: np.ndarray, directions: np.ndarray):
        """Closest hits: (instance, primitive, t, alpha_geom, position)."""
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(directions, np.float32).reshape(-1, 3)
        n = o.shape[0]
        inst, prim = np.zeros(n, np.int32), np.zeros(n, np.int32)
        t, a, p = np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros((n, 3), np.float32)
        rc = self._lib.pale_trace_rays(self._h, n, o.ctypes.data_as(N.f32p), d.ctypes.data_as(N.f32p),
                                       inst.ctypes.data_as(N.i32p), prim.ctypes.data_as(N.i32p),
                                       t.ctypes.data_as(N.f32p), a.ctypes.data_as(N.f32p), p.ctypes.data_as(N.f32p))
        _check(self._lib, self._h, rc, "trace_rays")
        return inst, prim, t, a, p

    def trace_transmittance(self, origins: np.ndarray, directions: np.ndarray):
        """Transmit-mode queries: (mesh instance, world t, transmissivity of
        the surfel cloud along the ray)."""
        o = np.ascontiguousarray(origins, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(directions, np.float32).reshape(-1, 3)
        n = o.shape[0]
        inst, t, T = np.zeros(n, np.int32), np.zeros(n, np.float32), np.zeros(n, np.float32)
        rc = self._lib.pale_trace_transmittance(self._h, n, o.ctypes.data_as(N.f32p), d.ctypes.data_as(N.f32p),
                                                inst.ctypes.data_as(N.i32p), t.ctypes.data_as(N.f32p),
                                                T.ctypes.data_as(N.f32p))
        _check(self._lib, self._h, rc, "trace_transmittance")
        return inst, t, T

    def gather_irradiance(self, points: np.ndarray, normals: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        nm = np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
        E = np.zeros_like(x)
        rc = self._lib.pale_gather_irradiance(self._h, x.shape[0], x.ctypes.data_as(N.f32p),
                                              nm.ctypes.data_as(N.f32p), E.ctypes.data_as(N.f32p))
        _check(self._lib, self._h, rc, "gather_irradiance")
        return E

    def load_photons(self, position, power, direction):
        p = np.ascontiguousarray(position, np.float32).reshape(-1, 3)
        w = np.ascontiguousarray(power, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(direction, np.float32).reshape(-1, 3)
        rc = self._lib.pale_load_photons(self._h, p.shape[0], p.ctypes.data_as(N.f32p), w.ctypes.data_as(N.f32p),
                                         d.ctypes.data_as(N.f32p))
        _check(self._lib, self._h, rc, "load_photons")

    def get_photons(self):
        cnt = C.c_uint32()
        _check(self._lib, self._h, self._lib.pale_get_photons(self._h, C.byref(cnt), None, None, None, None,
                                                              None, None), "get_photons")
        n = int(cnt.value)
        pos, pw, dr = (np.zeros((max(1, n), 3), np.float32) for _ in range(3))
        cid, srt = np.zeros(max(1, n), np.uint32), np.zeros(max(1, n), np.uint32)
        gi = np.zeros(7, np.float32)
        rc = self._lib.pale_get_photons(self._h, C.byref(cnt), pos.ctypes.data_as(N.f32p), pw.ctypes.data_as(N.f32p),
                                        dr.ctypes.data_as(N.f32p), cid.ctypes.data_as(N.u32p),
                                        srt.ctypes.data_as(N.u32p), gi.ctypes.data_as(N.f32p))
        _check(self._lib, self._h, rc, "get_photons")
        return dict(position=pos[:n], power=pw[:n], direction=dr[:n], cell_id=cid[:n], sorted=srt[:n], grid=gi)

    def get_bvh(self):
        n = self.num_points
        cnt = C.c_uint32()
        _check(self._lib, self._h, self._lib.pale_get_bvh(self._h, None, C.byref(cnt), None, 0), "get_bvh")
        codes = np.zeros(max(1, n), np.uint32)
        nodes = np.zeros((max(1, cnt.value), 16), np.float32)
        rc = self._lib.pale_get_bvh(self._h, codes.ctypes.data_as(N.u32p), C.byref(cnt),
                                    nodes.ctypes.data_as(N.f32p), cnt.value)
        _check(self._lib, self._h, rc, "get_bvh")
        return codes[:n], nodes[: cnt.value]
