"""numpy restatement of the device density control (test infrastructure).

prune_indices follows compute_prune_indices_by_opacity
(python/density_control.py:199-263) and split follows
densify_points_long_axis_split (:6-196) followed by remove_points(parents)
and add_points(children) (pale_bindings.cpp:1081-1395); both break ties by
the lower index, where the reference's default argsort leaves them in no
defined order.  Pinned against the reference itself by
tests/golden/density_steps.npz.
"""
from __future__ import annotations

from typing import Dict, Optional

import numpy as np

FIELDS = ("position", "tangent_u", "tangent_v", "scale", "albedo", "opacity", "beta")


def prune_indices(opa: np.ndarray, min_opacity: float, use_quantile: bool, max_fraction: float,
                  min_keep: int) -> np.ndarray:
    n = opa.shape[0]
    if n == 0:
        return np.zeros(0, np.int64)
    thr = float(np.quantile(opa, min(1.0, max(0.0, float(min_opacity))))) if use_quantile else float(min_opacity)
    cand = np.nonzero(opa <= thr)[0]
    cap = min(int(max_fraction * n), max(0, n - min_keep))
    if cand.size == 0 or cap <= 0:
        return np.zeros(0, np.int64)
    if cand.size > cap:
        cand = cand[np.argsort(opa[cand], kind="stable")[:cap]]
    return np.sort(cand).astype(np.int64)


def split(p: Dict[str, np.ndarray], importance: Optional[np.ndarray] = None, max_new_points: Optional[int] = None,
          split_distance: float = 0.6, minor_axis_shrink: float = 0.85, opacity_reduction: float = 0.6,
          min_long_axis_scale: float = 0.0, grad_threshold: float = 0.0):
    """Returns (parents, children dict)."""
    empty = (np.zeros(0, np.int64), None)
    sc = p["scale"]
    lng = np.maximum(sc[:, 0], sc[:, 1])
    cand = np.nonzero(lng >= min_long_axis_scale)[0]
    score = importance[cand] if importance is not None else None
    if importance is not None and grad_threshold > 0.0:
        keep = score >= grad_threshold
        cand, score = cand[keep], score[keep]
    if cand.size == 0:
        return empty
    if max_new_points is not None:
        mp = max_new_points // 2
        if mp <= 0:
            return empty
        if cand.size > mp:
            key = score if score is not None else lng[cand]
            cand = cand[np.argsort(-key, kind="stable")[:mp]]
    parents = np.unique(cand).astype(np.int64)
    out = {k: [] for k in FIELDS}
    for i in parents:
        su, sv = float(sc[i, 0]), float(sc[i, 1])
        long_u = su >= sv
        lo, sh = (su, sv) if long_u else (sv, su)
        axis = p["tangent_u"][i] if long_u else p["tangent_v"][i]
        off = np.float32(split_distance * (3.0 * lo)) * axis
        cl, cs = lo * (1.0 - split_distance), sh * minor_axis_shrink
        child_scale = np.array([cl, cs] if long_u else [cs, cl], np.float32)
        op = float(np.clip(float(p["opacity"][i]) * opacity_reduction, 0.0, 1.0))
        for pos in (p["position"][i] + off, p["position"][i] - off):
            out["position"].append(pos)
            out["tangent_u"].append(p["tangent_u"][i])
            out["tangent_v"].append(p["tangent_v"][i])
            out["scale"].append(child_scale)
            out["albedo"].append(p["albedo"][i])
            out["opacity"].append(op)
            out["beta"].append(float(p["beta"][i]))
    return parents, {k: np.asarray(v, np.float32) for k, v in out.items()}


def apply_split(p: Dict[str, np.ndarray], parents: np.ndarray, children: Dict[str, np.ndarray]):
    """remove_points(parents) then add_points(children)."""
    keep = np.ones(p["position"].shape[0], bool)
    keep[parents] = False
    return {k: np.concatenate([p[k][keep], children[k]]) for k in FIELDS}
