"""ctypes view of the C-ABI in include/pale_b200.h.

The renderer lives in ``libpale_b200.so`` next to this file (built by
``__graft_entry__.build()`` or ``python -m differentiablepointrendering_b200.build``).
There is no fallback: importing the product without the library raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional, Sequence

import numpy as np

from .scene import POINT_FIELDS, SceneArrays, as_points

LIB_NAME = "libpale_b200.so"

f32p = C.POINTER(C.c_float)
u32p = C.POINTER(C.c_uint32)
i32p = C.POINTER(C.c_int32)


class PaleSettings(C.Structure):
    _fields_ = [("photons_per_launch", C.c_uint32), ("max_bounces", C.c_uint32),
                ("forward_passes", C.c_uint32), ("gather_passes", C.c_uint32),
                ("adjoint_bounces", C.c_uint32), ("adjoint_passes", C.c_uint32),
                ("seed", C.c_uint64), ("random_number", C.c_uint32), ("rr_start", C.c_uint32),
                ("q_null", C.c_float), ("q_reflect", C.c_float), ("q_transmit", C.c_float),
                ("gather_radius", C.c_float), ("leaf_size", C.c_uint32), ("rng_mode", C.c_uint32),
                ("debug_images", C.c_uint32), ("exposure", C.c_float), ("gamma", C.c_float),
                ("null_weight", C.c_uint32), ("gradients", C.c_uint32), ("camera_seeds", C.c_uint32),
                ("gather_batch_paths", C.c_uint32), ("adjoint_batch_paths", C.c_uint32),
                ("walk_block", C.c_uint32), ("estimator", C.c_uint32), ("vertex_store", C.c_uint32),
                ("vertex_store_bytes", C.c_uint64)]


class PaleView(C.Structure):
    _fields_ = [("scene", C.c_uint32), ("camera", C.c_uint32), ("passes", C.c_uint32), ("depth", C.c_uint32),
                ("first_pass", C.c_uint32), ("pass_count", C.c_uint32)]


class PalePoints(C.Structure):
    _fields_ = [("count", C.c_uint32)] + [(k, f32p) for k in POINT_FIELDS]


class PaleSceneDesc(C.Structure):
    _fields_ = [("num_vertices", C.c_uint32), ("vertices", f32p),
                ("num_triangles", C.c_uint32), ("triangles", u32p),
                ("num_meshes", C.c_uint32), ("mesh_ranges", u32p),
                ("num_materials", C.c_uint32), ("materials", f32p),
                ("num_instances", C.c_uint32), ("instance_mesh", u32p), ("instance_material", u32p),
                ("instance_object_to_world", f32p), ("instance_world_to_object", f32p),
                ("num_cameras", C.c_uint32), ("camera_inv_view", f32p), ("camera_forward", f32p),
                ("camera_fovy_deg", f32p), ("camera_size", u32p), ("camera_names", C.c_char_p),
                ("points", PalePoints)]


class PaleStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in (
        "photon_segments", "gather_segments", "adjoint_segments", "photons_stored", "gradient_events",
        "gather_queries", "node_visits", "surfel_tests", "photons_scanned", "gather_node_visits",
        "gather_surfel_tests", "gather_photons_scanned", "kernel_launches")] + \
        [(k, C.c_float) for k in ("forward_ms", "backward_ms", "photon_ms", "gather_ms")] + \
        [("timed_ms", C.c_float * 4), ("timed_launches", C.c_uint32 * 4), ("vertex_bytes", C.c_uint64),
         ("vertex_chunks_stored", C.c_uint32), ("vertex_chunks_replayed", C.c_uint32),
         ("vertex_records", C.c_uint64), ("vertex_entries", C.c_uint64)]

    TIMED = ("trace", "lookup", "adjoint_bounce", "transport")

    def as_dict(self) -> Dict[str, float]:
        out = {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("timed")}
        for i, name in enumerate(self.TIMED):
            out[f"{name}_ms"] = float(self.timed_ms[i])
            out[f"{name}_launches"] = int(self.timed_launches[i])
        return out


class PaleOptimizer(C.Structure):
    _fields_ = [("type", C.c_uint32), ("flags", C.c_uint32), ("lr", C.c_double * 6), ("beta1", C.c_double),
                ("beta2", C.c_double), ("eps", C.c_double), ("momentum", C.c_double),
                ("opacity_reset", C.c_float), ("reference_dir", C.c_float * 3)]


OPT_ADAM, OPT_SGD, OPT_MASKED_ADAM = 0, 1, 2
OPT_SURFEL_MASK = 1
OPTIMIZER_TYPES = {"adam": OPT_ADAM, "sgd": OPT_SGD, "masked_adam": OPT_MASKED_ADAM,
                   "nullgrad_adam": OPT_MASKED_ADAM, "sparse_adam": OPT_MASKED_ADAM}
# Learning-rate keys of OptimizationConfig (python/config.py:46-51) with
# their defaults, in the group order of create_optimizer.
LR_KEYS = (("learning_rate_position", 1.6e-4), ("learning_rate_tangent", 1.0e-3),
           ("learning_rate_scale", 5.0e-3), ("learning_rate_albedo", 2.5e-3),
           ("learning_rate_opacity", 5.0e-2), ("learning_rate_beta", 5.0e-2))


def optimizer_from_config(cfg: Optional[dict] = None, opacity_reset: Optional[float] = None) -> PaleOptimizer:
    """pale_optimizer from OptimizationConfig-style keys: optimizer_type,
    learning_rate_*, plus betas / eps / momentum (torch defaults, SGD
    momentum 0.8 as optimizers.py:62), surfel_mask (MaskedAdam with
    per-surfel masks) and reference_dir (tangent-frame orientation, +Z)."""
    cfg = dict(cfg or {})
    o = PaleOptimizer()
    name = str(cfg.pop("optimizer_type", "adam")).lower()
    if name not in OPTIMIZER_TYPES:
        raise ValueError(f"Unknown optimizer_type: {name}")
    o.type = OPTIMIZER_TYPES[name]
    o.flags = OPT_SURFEL_MASK if cfg.pop("surfel_mask", False) else 0
    for g, (key, default) in enumerate(LR_KEYS):
        o.lr[g] = float(cfg.pop(key, default))
    b1, b2 = cfg.pop("betas", (0.9, 0.999))
    o.beta1, o.beta2 = float(b1), float(b2)
    o.eps = float(cfg.pop("eps", 1e-8))
    o.momentum = float(cfg.pop("momentum", 0.8))
    o.opacity_reset = -1.0 if opacity_reset is None else float(opacity_reset)
    ref = cfg.pop("reference_dir", (0.0, 0.0, 1.0))
    for c in range(3):
        o.reference_dir[c] = float(ref[c])
    if cfg:
        raise ValueError(f"Unknown optimizer keys: {sorted(cfg)}")
    return o


# Settings-dict keys of the reference (pale_bindings.cpp:123-139) plus the
# ones this build exposes that the reference hard-codes.
SETTINGS_KEYS = {
    "photons": "photons_per_launch", "bounces": "max_bounces", "forward_passes": "forward_passes",
    "gather_passes": "gather_passes", "adjoint_bounces": "adjoint_bounces",
    "adjoint_passes": "adjoint_passes", "seed": "seed", "random_number": "random_number",
    "rr_start": "rr_start", "q_null": "q_null", "q_reflect": "q_reflect", "q_transmit": "q_transmit",
    "gather_radius": "gather_radius", "leaf_size": "leaf_size", "debug_images": "debug_images",
    "exposure": "exposure", "gamma": "gamma",
    "gather_batch_paths": "gather_batch_paths", "adjoint_batch_paths": "adjoint_batch_paths",
    "walk_block": "walk_block", "vertex_store_bytes": "vertex_store_bytes",
}
IGNORED_KEYS = ("logging", "depth_distort_weight", "normal_consistency_weight")


def default_settings(lib=None) -> PaleSettings:
    s = PaleSettings()
    s.photons_per_launch, s.max_bounces, s.forward_passes, s.gather_passes = 1000000, 6, 6, 6
    s.adjoint_bounces, s.adjoint_passes, s.seed, s.random_number, s.rr_start = 6, 6, 42, 42, 6
    s.q_null, s.q_reflect, s.q_transmit, s.gather_radius = 0.5, 0.5, 0.0, 0.01
    s.leaf_size, s.rng_mode, s.debug_images, s.exposure, s.gamma = 1, 0, 0, 1.0, 2.2
    return s


def settings_from_dict(d: Optional[dict]) -> PaleSettings:
    s = default_settings()
    for k, v in (d or {}).items():
        if k in IGNORED_KEYS:
            continue
        if k == "rng_mode":
            s.rng_mode = {"reference": 0, "decorrelated": 1}.get(v, v) if isinstance(v, str) else int(v)
            continue
        if k == "null_weight":
            s.null_weight = {"reference": 0, "unbiased": 1}.get(v, v) if isinstance(v, str) else int(v)
            continue
        if k == "gradients":
            s.gradients = {"opacity": 0, "all": 1}.get(v, v) if isinstance(v, str) else int(v)
            continue
        if k == "camera_seeds":
            s.camera_seeds = {"selection": 0, "camera": 1}.get(v, v) if isinstance(v, str) else int(v)
            continue
        if k == "estimator":
            s.estimator = {"reference": 0, "gather": 1}.get(v, v) if isinstance(v, str) else int(v)
            continue
        if k == "vertices":
            s.vertex_store = {"auto": 0, "checkpoint": 1, "replay": 2}.get(v, v) if isinstance(v, str) else int(v)
            continue
        if k not in SETTINGS_KEYS:
            raise KeyError(f"unknown renderer setting '{k}'")
        field = SETTINGS_KEYS[k]
        cur = getattr(s, field)
        setattr(s, field, float(v) if isinstance(cur, float) else int(v))
    return s


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


class PointsHolder:
    """Keeps contiguous float32 arrays alive behind a PalePoints struct."""

    def __init__(self, pts: Optional[Dict[str, np.ndarray]] = None, n: int = 0, alloc: bool = False):
        if pts is None:
            from .scene import empty_points
            pts = empty_points(n)
        self.arrays = as_points(pts) if not alloc else pts
        self.struct = PalePoints()
        self.struct.count = int(self.arrays["position"].shape[0])
        for k in POINT_FIELDS:
            setattr(self.struct, k, _ptr(self.arrays[k], f32p))


class SceneDescHolder:
    """Builds a PaleSceneDesc from SceneArrays and keeps its buffers alive."""

    def __init__(self, sc: SceneArrays, struct_cls=PaleSceneDesc, points_cls=PalePoints):
        c = lambda a, dt: np.ascontiguousarray(a, dt)
        self.v = c(sc.vertices, np.float32)
        self.t = c(sc.triangles, np.uint32)
        self.mr = c(sc.mesh_ranges, np.uint32)
        self.mat = c(sc.materials, np.float32)
        self.im = c(sc.instance_mesh, np.uint32)
        self.imat = c(sc.instance_material, np.uint32)
        self.o2w = c(sc.object_to_world, np.float32)
        self.w2o = c(sc.world_to_object, np.float32)
        self.civ = c(sc.camera_inv_view, np.float32)
        self.cf = c(sc.camera_forward, np.float32)
        self.fov = c(sc.camera_fovy, np.float32)
        self.csz = c(sc.camera_size, np.uint32)
        names = b"".join(n.encode()[:15].ljust(16, b"\0") for n in sc.camera_names)
        self.names = C.create_string_buffer(names, max(1, len(names)))
        self.points = PointsHolder(sc.points)
        d = struct_cls()
        d.num_vertices, d.vertices = self.v.shape[0], _ptr(self.v, f32p)
        d.num_triangles, d.triangles = self.t.shape[0], _ptr(self.t, u32p)
        d.num_meshes, d.mesh_ranges = self.mr.shape[0], _ptr(self.mr, u32p)
        d.num_materials, d.materials = self.mat.shape[0], _ptr(self.mat, f32p)
        d.num_instances = self.im.shape[0]
        d.instance_mesh, d.instance_material = _ptr(self.im, u32p), _ptr(self.imat, u32p)
        d.instance_object_to_world, d.instance_world_to_object = _ptr(self.o2w, f32p), _ptr(self.w2o, f32p)
        d.num_cameras = self.civ.shape[0]
        d.camera_inv_view, d.camera_forward = _ptr(self.civ, f32p), _ptr(self.cf, f32p)
        d.camera_fovy_deg, d.camera_size = _ptr(self.fov, f32p), _ptr(self.csz, u32p)
        d.camera_names = C.cast(self.names, C.c_char_p)
        p = points_cls()
        p.count = self.points.struct.count
        for k in POINT_FIELDS:
            setattr(p, k, getattr(self.points.struct, k))
        d.points = p
        self.struct = d


_LIB = None


def library_path() -> str:
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)


def load_library() -> C.CDLL:
    """Loads the CUDA library; raises if it was not built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.isfile(path):
        raise RuntimeError(f"{LIB_NAME} is missing at {path}; build it with "
                           "`python -m differentiablepointrendering_b200.build`")
    lib = C.CDLL(path)
    H = C.c_void_p
    sig = {
        "pale_default_settings": (None, [C.POINTER(PaleSettings)]),
        "pale_version": (C.c_char_p, []),
        "pale_last_error": (C.c_char_p, [H]),
        "pale_create": (C.c_int, [C.POINTER(PaleSceneDesc), C.POINTER(PaleSettings), C.POINTER(H)]),
        "pale_destroy": (C.c_int, [H]),
        "pale_point_count": (C.c_int, [H, u32p]),
        "pale_camera_count": (C.c_int, [H, u32p]),
        "pale_camera_info": (C.c_int, [H, C.c_uint32, C.c_char_p, u32p, u32p]),
        "pale_render_forward": (C.c_int, [H, C.c_uint32, u32p, f32p, f32p]),
        "pale_render_gather": (C.c_int, [H, C.c_uint32, u32p, f32p, f32p]),
        "pale_render_forward_device": (C.c_int, [H, C.c_uint32, u32p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "pale_render_backward": (C.c_int, [H, C.c_uint32, u32p, f32p, C.POINTER(PalePoints), f32p]),
        "pale_render_backward_device": (C.c_int, [H, C.c_uint32, u32p, C.c_void_p, C.POINTER(PalePoints),
                                                  C.c_void_p]),
        "pale_get_points": (C.c_int, [H, C.POINTER(PalePoints)]),
        "pale_get_order": (C.c_int, [H, u32p]),
        "pale_apply_points": (C.c_int, [H, C.POINTER(PalePoints)]),
        "pale_apply_points_device": (C.c_int, [H, C.POINTER(PalePoints), C.c_void_p]),
        "pale_rebuild": (C.c_int, [H, C.POINTER(PalePoints)]),
        "pale_get_asset": (C.c_int, [H, C.POINTER(PalePoints)]),
        "pale_render_forward_loss": (C.c_int, [H, C.c_uint32, u32p, f32p, C.c_uint32, f32p, f32p, f32p,
                                               C.POINTER(C.c_double)]),
        "pale_render_forward_loss_device": (C.c_int, [H, C.c_uint32, u32p, C.c_void_p, C.c_uint32, C.c_void_p,
                                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "pale_optimizer_step": (C.c_int, [H, C.POINTER(PaleOptimizer), C.POINTER(PalePoints), C.c_void_p]),
        "pale_optimizer_reset": (C.c_int, [H]),
        "pale_prune_by_opacity": (C.c_int, [H, C.c_float, C.c_uint32, C.c_double, C.c_uint32, u32p,
                                            C.POINTER(C.c_int64)]),
        "pale_densify_long_axis_split": (C.c_int, [H, C.c_void_p, C.c_int64, C.c_double, C.c_double, C.c_double,
                                                   C.c_float, C.c_float, u32p, C.POINTER(C.c_int64)]),
        "pale_trace_rays": (C.c_int, [H, C.c_uint32, f32p, f32p, i32p, i32p, f32p, f32p, f32p]),
        "pale_trace_transmittance": (C.c_int, [H, C.c_uint32, f32p, f32p, i32p, f32p, f32p]),
        "pale_gather_irradiance": (C.c_int, [H, C.c_uint32, f32p, f32p, f32p]),
        "pale_load_photons": (C.c_int, [H, C.c_uint32, f32p, f32p, f32p]),
        "pale_get_photons": (C.c_int, [H, u32p, f32p, f32p, f32p, u32p, u32p, f32p]),
        "pale_get_bvh": (C.c_int, [H, u32p, u32p, f32p, C.c_uint32]),
        "pale_get_stats": (C.c_int, [H, C.POINTER(PaleStats)]),
        "pale_build_lbvh_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                              C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_void_p]),
        "pale_lbvh_node_count": (C.c_uint32, [C.c_uint32, C.c_uint32]),
        "pale_trace_photon_map": (C.c_int, [C.c_void_p, C.c_void_p]),
        "pale_render_views_loss_device": (C.c_int, [C.c_uint32, C.POINTER(C.c_void_p), C.c_int, C.c_uint32,
                                                    C.POINTER(PaleView), C.c_void_p, C.c_uint32, C.c_void_p,
                                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "pale_render_views_backward_device": (C.c_int, [C.c_uint32, C.POINTER(C.c_void_p), C.c_uint32,
                                                        C.POINTER(PaleView), C.c_void_p, C.POINTER(PalePoints),
                                                        C.c_void_p]),
        "pale_render_views_gradients_device": (C.c_int, [C.c_uint32, C.POINTER(C.c_void_p), C.c_uint32,
                                                         C.POINTER(PaleView), C.c_void_p, C.POINTER(PalePoints),
                                                         C.c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


EXPORTED = ("pale_default_settings", "pale_version", "pale_last_error", "pale_create", "pale_destroy",
            "pale_point_count", "pale_camera_count", "pale_camera_info", "pale_render_forward", "pale_render_gather",
            "pale_render_forward_device", "pale_render_backward", "pale_render_backward_device",
            "pale_get_points", "pale_get_order", "pale_apply_points", "pale_rebuild", "pale_trace_rays",
            "pale_trace_transmittance", "pale_gather_irradiance", "pale_load_photons", "pale_get_photons", "pale_get_bvh",
            "pale_get_stats", "pale_build_lbvh_noalloc", "pale_get_asset", "pale_optimizer_step",
            "pale_optimizer_reset", "pale_render_forward_loss", "pale_render_forward_loss_device",
            "pale_prune_by_opacity", "pale_densify_long_axis_split", "pale_apply_points_device",
            "pale_lbvh_node_count", "pale_render_views_loss_device", "pale_render_views_backward_device",
            "pale_trace_photon_map", "pale_render_views_gradients_device")
NOALLOC_MAX_SURFELS = 16384


def cams_array(idx: Sequence[int]) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(list(idx), np.uint32))
