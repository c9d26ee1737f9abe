"""ctypes wrapper of the CPU oracle (oracle/pale_oracle.c) for the tests.

The oracle is the checker: tests compare the CUDA renderer against it.  Its
struct layouts equal the C-ABI's, so the same ctypes classes are reused.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
from typing import Dict, List, Optional

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

from build_oracle import build_oracle  # noqa: E402
from differentiablepointrendering_b200 import _native as N  # noqa: E402
from differentiablepointrendering_b200.scene import POINT_FIELDS, SceneArrays, as_points  # noqa: E402

_LIB = None


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        L = C.CDLL(build_oracle())
        P = C.c_void_p
        sig = {
            "orc_create": (P, [C.POINTER(N.PaleSceneDesc), C.POINTER(N.PaleSettings), C.c_int]),
            "orc_destroy": (None, [P]),
            "orc_set_threads": (None, [C.c_int]),
            "orc_point_count": (C.c_uint32, [P]),
            "orc_get_order": (C.c_int, [P, N.u32p]),
            "orc_get_points": (C.c_int, [P, C.POINTER(N.PalePoints)]),
            "orc_apply_points": (C.c_int, [P, C.POINTER(N.PalePoints)]),
            "orc_rebuild": (C.c_int, [P, C.POINTER(N.PalePoints)]),
            "orc_render_forward": (C.c_int, [P, C.c_uint32, N.u32p, N.f32p, N.f32p]),
            "orc_render_gather": (C.c_int, [P, C.c_uint32, N.u32p, N.f32p, N.f32p]),
            "orc_render_backward": (C.c_int, [P, C.c_uint32, N.u32p, N.f32p, C.POINTER(N.PalePoints), N.f32p]),
            "orc_render_forward_views": (C.c_int, [P, C.c_uint32, N.u32p, N.u32p, N.f32p, N.f32p]),
            "orc_render_backward_views": (C.c_int, [P, C.c_uint32, N.u32p, N.u32p, N.u32p, N.f32p,
                                                    C.POINTER(N.PalePoints)]),
            "orc_trace_rays": (C.c_int, [P, C.c_uint32, N.f32p, N.f32p, N.i32p, N.i32p, N.f32p, N.f32p, N.f32p]),
            "orc_trace_transmittance": (C.c_int, [P, C.c_uint32, N.f32p, N.f32p, N.i32p, N.f32p, N.f32p]),
            "orc_gather_irradiance": (C.c_int, [P, C.c_uint32, N.f32p, N.f32p, N.f32p]),
            "orc_load_photons": (C.c_int, [P, C.c_uint32, N.f32p, N.f32p, N.f32p]),
            "orc_get_photons": (C.c_int, [P, N.u32p, N.f32p, N.f32p, N.f32p, N.u32p, N.u32p, N.f32p]),
            "orc_get_stats": (C.c_int, [P, C.POINTER(N.PaleStats)]),
            "orc_lbvh_build": (C.c_uint32, [C.c_uint32, N.f32p, N.f32p, N.f32p, C.c_uint32, C.c_uint32, N.u32p,
                                            N.u32p, N.f32p, C.c_uint32]),
            "orc_surfel_aabbs": (None, [C.c_uint32, N.f32p, N.f32p, N.f32p, N.f32p, N.f32p, N.f32p]),
            "orc_per_item_seed": (C.c_uint64, [C.c_uint64, C.c_uint64]),
            "orc_xorshift_floats": (None, [C.c_uint64, C.c_uint32, N.f32p]),
            "orc_xorshift128_raw": (None, [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, N.u32p]),
            "orc_mt19937_64": (None, [C.c_uint64, C.c_uint32, C.POINTER(C.c_uint64)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def fptr(a):
    return a.ctypes.data_as(N.f32p)


def uptr(a):
    return a.ctypes.data_as(N.u32p)


class OracleRenderer:
    """Same surface as pale.Renderer (the subset the tests use) on the CPU
    oracle.  bvh_kind 0 = reference median split, 1 = LBVH restatement."""

    def __init__(self, scene: SceneArrays, settings: Optional[dict] = None, bvh_kind: int = 0, threads: int = 0):
        self.L = lib()
        self.scene = scene
        self.settings = N.settings_from_dict(settings)
        self._desc = N.SceneDescHolder(scene)
        if threads:
            self.L.orc_set_threads(threads)
        self.h = self.L.orc_create(C.byref(self._desc.struct), C.byref(self.settings), bvh_kind)
        if not self.h:
            raise RuntimeError("orc_create failed")
        self.names = list(scene.camera_names)
        self.sizes = [(int(w), int(h)) for w, h in scene.camera_size]

    def close(self):
        if self.h:
            self.L.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @property
    def num_points(self) -> int:
        return int(self.L.orc_point_count(self.h))

    def render_forward(self, camera_name="") -> Dict[str, np.ndarray]:
        """One camera by name, a list of names, or every camera ("")."""
        return self._render(camera_name, self.L.orc_render_forward)

    def render_gather(self, camera_name="") -> Dict[str, np.ndarray]:
        return self._render(camera_name, self.L.orc_render_gather)

    def _render(self, camera_name, fn) -> Dict[str, np.ndarray]:
        want = [camera_name] if isinstance(camera_name, str) else list(camera_name)
        idx = [i for i, n in enumerate(self.names) if (want == [""] or n in want)]
        pix = sum(self.sizes[i][0] * self.sizes[i][1] for i in idx)
        ldr = np.empty(max(1, pix) * 4, np.float32)
        raw = np.empty(max(1, pix) * 4, np.float32)
        cams = np.asarray(idx, np.uint32)
        assert fn(self.h, len(idx), uptr(cams), fptr(ldr), fptr(raw)) == 0
        out, off = {}, 0
        for i in idx:
            w, h = self.sizes[i]
            n = w * h * 4
            out[self.names[i]] = ldr[off:off + n].reshape(h, w, 4).copy()
            out[self.names[i] + "_raw"] = raw[off:off + n].reshape(h, w, 4).copy()
            off += n
        return out

    def render_backward(self, targetRgb32f: Dict[str, np.ndarray]):
        idx, imgs = [], []
        for i, name in enumerate(self.names):
            if name in targetRgb32f and bool(self.scene.camera_adjoint[i]):
                a = np.asarray(targetRgb32f[name], np.float32)
                rgba = np.ones(a.shape[:2] + (4,), np.float32)
                rgba[..., :3] = a
                idx.append(i)
                imgs.append(rgba)
        grads = N.PointsHolder(n=self.num_points)
        dldi = np.concatenate([im.reshape(-1) for im in imgs]) if imgs else np.zeros(4, np.float32)
        pix = sum(im.size for im in imgs)
        dbg = np.zeros(max(4, pix), np.float32)
        cams = np.asarray(idx, np.uint32)
        assert self.L.orc_render_backward(self.h, len(idx), uptr(cams), fptr(dldi), C.byref(grads.struct),
                                          fptr(dbg)) == 0
        g = {k: grads.arrays[k].copy() for k in POINT_FIELDS}
        return g, {"debug_opacity": dbg[:pix]}

    def render_views(self, cams, passes):
        """Forward render of cameras `cams` (indices) with passes[i] gather
        passes each: {name: LDR, name + "_raw": RAW} per view."""
        cams = np.asarray(cams, np.uint32)
        ps = np.asarray(passes, np.uint32)
        pix = sum(self.sizes[i][0] * self.sizes[i][1] for i in cams)
        ldr = np.empty(max(1, pix) * 4, np.float32)
        raw = np.empty(max(1, pix) * 4, np.float32)
        assert self.L.orc_render_forward_views(self.h, len(cams), uptr(cams), uptr(ps), fptr(ldr), fptr(raw)) == 0
        out, off = [], 0
        for i in cams:
            w, h = self.sizes[i]
            n = w * h * 4
            out.append((ldr[off:off + n].reshape(h, w, 4).copy(), raw[off:off + n].reshape(h, w, 4).copy()))
            off += n
        return out

    def backward_views(self, cams, passes, depths, dldi_rgb):
        """Adjoint of the views (passes and bounces per view, depth 0 = the
        settings') with dL/dI images (H, W, 3) per view; gradient dict."""
        cams = np.asarray(cams, np.uint32)
        ps = np.asarray(passes, np.uint32)
        ds = np.asarray(depths, np.uint32)
        parts = []
        for a in dldi_rgb:
            rgba = np.ones(a.shape[:2] + (4,), np.float32)
            rgba[..., :3] = a
            parts.append(rgba.reshape(-1))
        dl = np.concatenate(parts) if parts else np.zeros(4, np.float32)
        grads = N.PointsHolder(n=self.num_points)
        assert self.L.orc_render_backward_views(self.h, len(cams), uptr(cams), uptr(ps), uptr(ds), fptr(dl),
                                                C.byref(grads.struct)) == 0
        return {k: grads.arrays[k].copy() for k in POINT_FIELDS}

    def get_point_parameters(self):
        out = N.PointsHolder(n=self.num_points)
        self.L.orc_get_points(self.h, C.byref(out.struct))
        return {k: out.arrays[k].copy() for k in POINT_FIELDS}

    def get_point_order(self):
        o = np.zeros(max(1, self.num_points), np.uint32)
        self.L.orc_get_order(self.h, uptr(o))
        return o[: self.num_points]

    def apply_point_optimization(self, params):
        hold = N.PointsHolder(params)
        assert self.L.orc_apply_points(self.h, C.byref(hold.struct)) == 0

    def rebuild(self, asset_points):
        hold = N.PointsHolder(asset_points)
        assert self.L.orc_rebuild(self.h, C.byref(hold.struct)) == 0

    def trace_rays(self, o, d):
        o = np.ascontiguousarray(o, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(d, np.float32).reshape(-1, 3)
        n = o.shape[0]
        inst, prim = np.zeros(n, np.int32), np.zeros(n, np.int32)
        t, a, p = np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros((n, 3), np.float32)
        self.L.orc_trace_rays(self.h, n, fptr(o), fptr(d), inst.ctypes.data_as(N.i32p), prim.ctypes.data_as(N.i32p),
                              fptr(t), fptr(a), fptr(p))
        return inst, prim, t, a, p

    def trace_transmittance(self, o, d):
        o = np.ascontiguousarray(o, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(d, np.float32).reshape(-1, 3)
        n = o.shape[0]
        inst, t, T = np.zeros(n, np.int32), np.zeros(n, np.float32), np.zeros(n, np.float32)
        self.L.orc_trace_transmittance(self.h, n, fptr(o), fptr(d), inst.ctypes.data_as(N.i32p), fptr(t), fptr(T))
        return inst, t, T

    def gather_irradiance(self, pts, nrm):
        x = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
        nm = np.ascontiguousarray(nrm, np.float32).reshape(-1, 3)
        E = np.zeros_like(x)
        self.L.orc_gather_irradiance(self.h, x.shape[0], fptr(x), fptr(nm), fptr(E))
        return E

    def load_photons(self, pos, pw, dr):
        p = np.ascontiguousarray(pos, np.float32)
        w = np.ascontiguousarray(pw, np.float32)
        d = np.ascontiguousarray(dr, np.float32)
        self.L.orc_load_photons(self.h, p.shape[0], fptr(p), fptr(w), fptr(d))

    def get_photons(self):
        cnt = C.c_uint32()
        self.L.orc_get_photons(self.h, C.byref(cnt), None, None, None, None, None, None)
        n = int(cnt.value)
        pos, pw, dr = (np.zeros((max(1, n), 3), np.float32) for _ in range(3))
        cid, srt = np.zeros(max(1, n), np.uint32), np.zeros(max(1, n), np.uint32)
        gi = np.zeros(7, np.float32)
        self.L.orc_get_photons(self.h, C.byref(cnt), fptr(pos), fptr(pw), fptr(dr), uptr(cid), uptr(srt), fptr(gi))
        return dict(position=pos[:n], power=pw[:n], direction=dr[:n], cell_id=cid[:n], sorted=srt[:n], grid=gi)

    def stats(self):
        st = N.PaleStats()
        self.L.orc_get_stats(self.h, C.byref(st))
        return st.as_dict()


def lbvh_reference(positions, lo, hi, leaf_size=4, top=256):
    """Oracle LBVH restatement: (codes, order, nodes[count,16])."""
    L = lib()
    p = np.ascontiguousarray(positions, np.float32)
    l = np.ascontiguousarray(lo, np.float32)
    h = np.ascontiguousarray(hi, np.float32)
    n = p.shape[0]
    codes, order = np.zeros(max(1, n), np.uint32), np.zeros(max(1, n), np.uint32)
    cnt = L.orc_lbvh_build(n, fptr(p), fptr(l), fptr(h), leaf_size, top, uptr(codes), uptr(order), None, 0)
    nodes = np.zeros((max(1, cnt), 16), np.float32)
    L.orc_lbvh_build(n, fptr(p), fptr(l), fptr(h), leaf_size, top, None, None, fptr(nodes), cnt)
    return codes[:n], order[:n], nodes[:cnt]


def surfel_aabbs(pos, tu, tv, scale):
    L = lib()
    n = pos.shape[0]
    lo, hi = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32)
    args = [np.ascontiguousarray(a, np.float32) for a in (pos, tu, tv, scale)]
    L.orc_surfel_aabbs(n, *[fptr(a) for a in args], fptr(lo), fptr(hi))
    return lo, hi


def collected_asset_points(scene: SceneArrays):
    """Asset-order points after the reference's collection step
    (normalised tangents, clamped albedo/opacity), computed by the oracle."""
    o = OracleRenderer(scene, {"photons": 1, "forward_passes": 1}, bvh_kind=1)
    bvh = o.get_point_parameters()
    order = o.get_point_order()
    o.close()
    out = {}
    for k, v in bvh.items():
        a = np.empty_like(v)
        a[order] = v
        out[k] = a
    return out
