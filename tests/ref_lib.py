"""ctypes wrapper of oracle/_ref/libpale_ref.so: the reference renderer's own
kernel sources compiled for the CPU (test infrastructure).

The library is built from the reference checkout by oracle/build_ref.py; it
is only available where that checkout exists or where a built copy was
shipped (REFERENCE_CHECKOUT names the checkout; without it a built library
is used if present).  Tests that need it skip when it is absent.
"""
from __future__ import annotations

import ctypes as C
import os
import sys
from typing import Dict, Optional

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

from differentiablepointrendering_b200 import _native as N  # noqa: E402
from differentiablepointrendering_b200.scene import SceneArrays  # noqa: E402

LIB_PATH = os.path.join(ROOT, "oracle", "_ref", "libpale_ref.so")
_LIB = None


def checkout() -> Optional[str]:
    path = os.environ.get("REFERENCE_CHECKOUT")
    if path and os.path.isdir(os.path.join(path, "Pale", "Renderer", "Kernels")):
        return path
    return None


def available() -> bool:
    return checkout() is not None or os.path.exists(LIB_PATH)


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        ref = checkout()
        if ref is not None:
            from build_ref import build_ref
            build_ref(ref)
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(LIB_PATH)
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        u32p, f32p = N.u32p, N.f32p
        sig = {
            "ref_set_threads": (None, [C.c_int]),
            "ref_create": (P, [C.POINTER(N.PaleSceneDesc), C.POINTER(N.PaleSettings)]),
            "ref_destroy": (None, [P]),
            "ref_point_count": (C.c_uint32, [P]),
            "ref_get_order": (C.c_int, [P, u32p]),
            "ref_render_forward": (C.c_int, [P, C.c_uint32, u32p, f32p, f32p]),
            "ref_trace_photons": (C.c_int, [P]),
            "ref_count_gather_segments": (C.c_uint64, [P, C.c_uint32, u32p]),
            "ref_render_backward": (C.c_int, [P, C.c_uint32, u32p, f32p, f32p]),
            "ref_get_photons": (C.c_int, [P, u32p, f32p, f32p, f32p, u32p, u32p]),
            "ref_get_segments": (None, [P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
            "ref_get_times": (None, [P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def _f(a):
    return a.ctypes.data_as(N.f32p)


def _u(a):
    return a.ctypes.data_as(N.u32p)


class ReferenceRenderer:
    """The reference's kernels on the CPU, with the subset of the
    pale.Renderer surface the parity tests use (render_forward,
    render_backward with opacity gradients, photons, point order)."""

    def __init__(self, scene: SceneArrays, settings: Optional[dict] = None, threads: int = 1):
        self.L = lib()
        self.L.ref_set_threads(int(threads))
        self.scene = scene
        self.settings = N.settings_from_dict(settings)
        self._desc = N.SceneDescHolder(scene)
        self.h = self.L.ref_create(C.byref(self._desc.struct), C.byref(self.settings))
        if not self.h:
            raise RuntimeError("ref_create failed")
        self.names = list(scene.camera_names)
        self.sizes = [(int(w), int(h)) for w, h in scene.camera_size]

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @property
    def num_points(self) -> int:
        return int(self.L.ref_point_count(self.h))

    def _select(self, camera_name=""):
        return [i for i, n in enumerate(self.names) if (not camera_name or n == camera_name)]

    def render_forward(self, camera_name: str = "") -> Dict[str, np.ndarray]:
        idx = self._select(camera_name)
        pix = sum(self.sizes[i][0] * self.sizes[i][1] for i in idx)
        ldr = np.empty(max(1, pix) * 4, np.float32)
        raw = np.empty(max(1, pix) * 4, np.float32)
        cams = np.asarray(idx, np.uint32)
        assert self.L.ref_render_forward(self.h, len(idx), _u(cams), _f(ldr), _f(raw)) == 0
        out, off = {}, 0
        for i in idx:
            w, h = self.sizes[i]
            n = w * h * 4
            out[self.names[i]] = ldr[off:off + n].reshape(h, w, 4).copy()
            out[self.names[i] + "_raw"] = raw[off:off + n].reshape(h, w, 4).copy()
            off += n
        return out

    def count_gather_segments(self, camera_name: str = "") -> int:
        idx = self._select(camera_name)
        cams = np.asarray(idx, np.uint32)
        return int(self.L.ref_count_gather_segments(self.h, len(idx), _u(cams)))

    def trace_photons(self):
        assert self.L.ref_trace_photons(self.h) == 0

    def render_backward_opacity(self, targetRgb32f: Dict[str, np.ndarray]) -> np.ndarray:
        idx, imgs = [], []
        for i, name in enumerate(self.names):
            if name in targetRgb32f:
                a = np.asarray(targetRgb32f[name], np.float32)
                rgba = np.ones(a.shape[:2] + (4,), np.float32)
                rgba[..., :3] = a
                idx.append(i)
                imgs.append(rgba)
        dldi = np.concatenate([im.reshape(-1) for im in imgs]) if imgs else np.zeros(4, np.float32)
        g = np.zeros(max(1, self.num_points), np.float32)
        cams = np.asarray(idx, np.uint32)
        assert self.L.ref_render_backward(self.h, len(idx), _u(cams), _f(dldi), _f(g)) == 0
        return g[: self.num_points]

    def get_point_order(self) -> np.ndarray:
        o = np.zeros(max(1, self.num_points), np.uint32)
        self.L.ref_get_order(self.h, _u(o))
        return o[: self.num_points]

    def get_photons(self):
        cnt = C.c_uint32()
        self.L.ref_get_photons(self.h, C.byref(cnt), None, None, None, None, None)
        n = int(cnt.value)
        pos, pw, dr = (np.zeros((max(1, n), 3), np.float32) for _ in range(3))
        cid, srt = np.zeros(max(1, n), np.uint32), np.zeros(max(1, n), np.uint32)
        self.L.ref_get_photons(self.h, C.byref(cnt), _f(pos), _f(pw), _f(dr), _u(cid), _u(srt))
        return dict(position=pos[:n], power=pw[:n], direction=dr[:n], cell_id=cid[:n], sorted=srt[:n])

    def segments(self):
        a, b = C.c_uint64(), C.c_uint64()
        self.L.ref_get_segments(self.h, C.byref(a), C.byref(b))
        return int(a.value), int(b.value)

    def times_ms(self):
        """(photon pass + grid, camera gather + post-process, adjoint) of the last calls."""
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        self.L.ref_get_times(self.h, C.byref(a), C.byref(b), C.byref(c))
        return float(a.value), float(b.value), float(c.value)
