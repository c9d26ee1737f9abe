"""numpy restatement of the device optimizer step (test infrastructure).

Float32 operation by operation as the kernel evaluates it (no fused
multiply-add), so that the device step can be compared with it at any
size.  The reference semantics it restates: torch.optim.Adam / SGD
(optimizers.py:11-66), MaskedAdam (optimizers.py:70-214) with
compute_surfel_update_mask (:216-246), the opacity reset of
training.py:707-711 and verify_parameters_inplane (training.py:326-343:
render_hooks.py:32-258).  It is pinned against the reference's own code by
tests/golden/optimizer_steps.npz.
"""
from __future__ import annotations

import math
from typing import Dict, Optional

import numpy as np

f32 = np.float32
GROUP = {"position": 0, "tangent_u": 1, "tangent_v": 1, "scale": 2, "albedo": 3, "opacity": 4, "beta": 5}
LR_KEYS = ("learning_rate_position", "learning_rate_tangent", "learning_rate_scale", "learning_rate_albedo",
           "learning_rate_opacity", "learning_rate_beta")
FIELDS = ("position", "tangent_u", "tangent_v", "scale", "albedo", "opacity", "beta")


class OptimizerOracle:
    def __init__(self, cfg: dict, mask: bool = False, betas=(0.9, 0.999), eps=1e-8, momentum=0.8,
                 ref=(0.0, 0.0, 1.0)):
        self.kind = cfg.get("optimizer_type", "adam")
        self.mask = mask and self.kind != "adam" and self.kind != "sgd"
        self.lr = [cfg[k] for k in LR_KEYS]
        self.b1, self.b2, self.eps, self.mu = betas[0], betas[1], eps, momentum
        self.ref = np.asarray(ref, f32)
        self.t = 0
        self.m: Optional[Dict[str, np.ndarray]] = None

    def step(self, p: Dict[str, np.ndarray], g: Dict[str, np.ndarray], opacity_reset=None):
        if self.m is None:
            self.m = {k: np.zeros_like(p[k]) for k in FIELDS}
            self.v = {k: np.zeros_like(p[k]) for k in FIELDS}
            self.steps = np.zeros(p["opacity"].shape[0], np.uint32)
        self.t += 1
        n = p["opacity"].shape[0]
        out = {}
        if self.mask:
            sq = np.zeros(n, f32)
            for k in FIELDS:
                a = g[k].reshape(n, -1)
                s = a[:, 0] * a[:, 0]
                for c in range(1, a.shape[1]):
                    s = s + a[:, c] * a[:, c]
                sq = sq + s
            upd = sq != 0
            self.steps = self.steps + upd.astype(np.uint32)
            tf = self.steps.astype(f32)
            bc1 = f32(1) - np.power(f32(self.b1), tf)
            bc2 = f32(1) - np.power(f32(self.b2), tf)
            with np.errstate(divide="ignore", invalid="ignore"):
                rcp1 = f32(1) / np.maximum(bc1, f32(1e-12))
            bc2s = np.sqrt(bc2)
        t = float(self.t)
        bc1d = 1.0 - self.b1 ** t
        bc2d = 1.0 - self.b2 ** t
        for k in FIELDS:
            gi = GROUP[k]
            lr = f32(self.lr[gi])
            P, G, M, V = p[k], g[k], self.m[k], self.v[k]
            if self.kind == "sgd":
                buf = G.copy() if self.t == 1 else M * f32(self.mu) + G
                self.m[k] = buf
                out[k] = P + (-lr) * buf
                continue
            omb1, omb2 = f32(1.0 - self.b1), f32(1.0 - self.b2)
            if self.kind == "adam":
                mm = M + omb1 * (G - M)
                vv = V * f32(self.b2) + omb2 * G * G
            elif not self.mask:
                mm = M * f32(self.b1) + omb1 * G
                vv = V * f32(self.b2) + omb2 * G * G
            else:
                mm = M * f32(self.b1) + omb1 * G
                vv = V * f32(self.b2) + omb2 * (G * G)
                shp = (n,) + (1,) * (P.ndim - 1)
                w = upd.reshape(shp)
                mm = np.where(w, mm, M)
                vv = np.where(w, vv, V)
                self.m[k], self.v[k] = mm, vv
                with np.errstate(divide="ignore", invalid="ignore"):
                    denom = np.sqrt(vv) / bc2s.reshape(shp) + f32(self.eps)
                    new = P - (rcp1.reshape(shp) * lr) * (mm / denom)
                out[k] = np.where(w, new, P)
                continue
            self.m[k], self.v[k] = mm, vv
            denom = np.sqrt(vv) / f32(math.sqrt(bc2d)) + f32(self.eps)
            out[k] = P + f32(-(self.lr[gi] / bc1d)) * (mm / denom)
        if opacity_reset is not None:
            out["opacity"] = np.full_like(out["opacity"], f32(opacity_reset))
        out, self.condition = project(out, self.ref)
        return out


def project(p: Dict[str, np.ndarray], ref):
    """verify_parameters_inplane: tangent frame, then the clamps.  Also
    returns, per surfel, |tangent_v| / |its part orthogonal to tangent_u|:
    the factor by which rounding errors grow in the Gram-Schmidt step."""
    tu, tv = p["tangent_u"], p["tangent_v"]

    def norm(a):
        return np.sqrt(a[:, 0] * a[:, 0] + a[:, 1] * a[:, 1] + a[:, 2] * a[:, 2])

    def dot(a, b):
        return a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1] + a[:, 2] * b[:, 2]

    u = tu / np.maximum(norm(tu), f32(1e-8))[:, None]
    s = tv - dot(tv, u)[:, None] * u
    degenerate = dot(s, s) < f32(1e-6)
    cond = np.where(degenerate, 1.0, norm(tv).astype(np.float64) / np.maximum(norm(s), 1e-30))
    a = np.where((np.abs(u[:, 1]) < f32(0.9))[:, None], np.array([0, 1, 0], f32), np.array([1, 0, 0], f32))
    a = a - dot(a, u)[:, None] * u
    s = np.where(degenerate[:, None], a, s)
    w = s / np.maximum(norm(s), f32(1e-8))[:, None]
    nrm = np.stack([u[:, 1] * w[:, 2] - u[:, 2] * w[:, 1], u[:, 2] * w[:, 0] - u[:, 0] * w[:, 2],
                    u[:, 0] * w[:, 1] - u[:, 1] * w[:, 0]], 1)
    nrm = nrm / np.maximum(norm(nrm), f32(1e-8))[:, None]
    ref = np.asarray(ref, f32)
    flip = (nrm[:, 0] * ref[0] + nrm[:, 1] * ref[1] + nrm[:, 2] * ref[2]) < 0
    w = np.where(flip[:, None], -w, w)
    out = dict(p)
    out["tangent_u"], out["tangent_v"] = u.astype(f32), w.astype(f32)
    out["scale"] = np.clip(p["scale"], f32(0.01), f32(1.0))
    out["albedo"] = np.clip(p["albedo"], f32(0), f32(1))
    out["opacity"] = np.clip(p["opacity"], f32(0), f32(1))
    out["beta"] = np.clip(p["beta"], f32(-3), f32(1))
    return {k: v.astype(f32) for k, v in out.items()}, np.maximum(cond, 1.0)


def assert_close_to(got: Dict[str, np.ndarray], want: Dict[str, np.ndarray], condition: np.ndarray,
                    ulps: float = 64.0):
    """Parameters equal up to float32 rounding: |got - want| <= ulps *
    2^-24 * max(|want|, 1) per entry (every field is of order one, and the
    tangents are unit vectors whose components all carry the rounding of
    the norm), tangent_v scaled by the Gram-Schmidt condition of its surfel."""
    eps = 2.0 ** -24
    for k in FIELDS:
        g, w = got[k].astype(np.float64), want[k].astype(np.float64)
        tol = ulps * eps * np.maximum(np.abs(w), 1.0)
        if k == "tangent_v":
            tol = tol * condition[:, None]
        bad = np.abs(g - w) > tol
        assert not bad.any(), (k, int(bad.sum()), np.argwhere(bad)[:5].tolist(), float(np.abs(g - w).max()))
