"""Seeded inputs of the density-control fixtures (density_steps.npz).

Shared by make_density_golden.py, which runs the reference's
python/density_control.py on them, and by the tests, which regenerate the
inputs from the seeds.  Opacities are distinct (the reference breaks ties
with an unstable argsort) and so are the densification scores.
"""
from __future__ import annotations

import numpy as np

N_PRUNE = 200
N_SPLIT = 64
# (name, min_opacity, use_quantile, max_fraction_to_prune, min_points_to_keep)
PRUNE = (
    ("q10", 0.1, True, 0.3, 1),
    ("q50_capped", 0.5, True, 0.3, 1),
    ("q0", 0.0, True, 0.3, 1),
    ("q100_capped", 1.0, True, 0.25, 1),
    ("abs25", 0.25, False, 0.3, 1),
    ("abs90_keep", 0.9, False, 1.0, 150),
    ("abs_none", -0.5, False, 0.3, 1),
)
# (name, use importance, max_new_points or None, min_long_axis_scale, grad_threshold)
SPLIT = (
    ("all", False, None, 0.0, 0.0),
    ("long_budget", False, 20, 0.0, 0.0),
    ("min_long", False, None, 0.02, 0.0),
    ("score_budget", True, 16, 0.0, 0.0),
    ("score_threshold", True, None, 0.0, 0.5),
    ("score_threshold_budget", True, 9, 0.01, 0.3),
)
WIDTH = {"position": 3, "tangent_u": 3, "tangent_v": 3, "scale": 2, "albedo": 3, "opacity": 1, "beta": 1}
FIELDS = tuple(WIDTH)


def points(n: int, seed: int):
    rng = np.random.default_rng(seed)
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    a = np.where(np.abs(nrm[:, :1]) < 0.9, np.array([[1.0, 0, 0]]), np.array([[0, 1.0, 0]]))
    tu = np.cross(nrm, a)
    tu /= np.linalg.norm(tu, axis=1, keepdims=True)
    tv = np.cross(nrm, tu)
    p = {
        "position": rng.uniform(-0.4, 0.4, (n, 3)),
        "tangent_u": tu,
        "tangent_v": tv,
        "scale": np.exp(rng.normal(np.log(0.01), 0.3, (n, 2))),
        "albedo": rng.uniform(0.2, 0.9, (n, 3)),
        "opacity": (rng.permutation(n) + rng.uniform(0.05, 0.95, n)) / n,
        "beta": rng.uniform(-1, 1, n),
    }
    return {k: v.astype(np.float32) for k, v in p.items()}


def importance(n: int, seed: int):
    rng = np.random.default_rng(seed)
    return ((rng.permutation(n) + rng.uniform(0.05, 0.95, n)) / n).astype(np.float32)
