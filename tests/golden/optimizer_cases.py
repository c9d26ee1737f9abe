"""Seeded inputs of the optimizer-step fixtures (optimizer_steps.npz).

Shared by make_optimizer_golden.py, which runs the reference's optimizer
code on them, and by the tests, which regenerate them from the seed.
The parameter set covers the projection's branches: tangent pairs that
are parallel (the Gram-Schmidt fallback, with the primary tangent both off
and along the y axis), frames whose normal points away from +Z (the flip),
and scales, albedos, opacities and betas outside their ranges (the clamps).
Some surfels get an all-zero gradient in some steps (MaskedAdam's mask).
"""
from __future__ import annotations

import numpy as np

N = 128
STEPS = 3
# (name, optimizer_type, per-surfel mask, opacity reset value per step or None)
SCENARIOS = (
    ("adam", "adam", False, (None, 0.1, None)),
    ("sgd", "sgd", False, (None, None, None)),
    ("masked_adam", "masked_adam", False, (None, None, None)),
    ("masked_adam_mask", "masked_adam", True, (None, None, 0.1)),
)
# OptimizationConfig learning rates (python/config.py:46-51), scaled up so
# that the clamps and the frame projection act within three steps.
LR = {"learning_rate_position": 1.6e-2, "learning_rate_tangent": 0.2, "learning_rate_scale": 0.2,
      "learning_rate_albedo": 0.2, "learning_rate_opacity": 0.3, "learning_rate_beta": 0.5}
WIDTH = {"position": 3, "tangent_u": 3, "tangent_v": 3, "scale": 2, "albedo": 3, "opacity": 1, "beta": 1}
FIELDS = tuple(WIDTH)


def _shape(k, n):
    return (n, WIDTH[k]) if WIDTH[k] > 1 else (n,)


def initial_parameters(seed: int = 2024):
    rng = np.random.default_rng(seed)
    p = {
        "position": rng.normal(0.0, 0.5, (N, 3)),
        "tangent_u": rng.normal(0.0, 1.0, (N, 3)),
        "tangent_v": rng.normal(0.0, 1.0, (N, 3)),
        "scale": rng.uniform(0.0, 1.3, (N, 2)),
        "albedo": rng.uniform(-0.2, 1.2, (N, 3)),
        "opacity": rng.uniform(-0.2, 1.2, N),
        "beta": rng.uniform(-3.5, 1.5, N),
    }
    # parallel tangent pairs: Gram-Schmidt fallback (x / y axis choice)
    p["tangent_v"][0:6] = 2.5 * p["tangent_u"][0:6]
    p["tangent_u"][6:10] = [[0.02, 1.0, 0.01], [0.0, -3.0, 0.0], [0.1, 0.95, 0.0], [0.0, 0.5, 0.0]]
    p["tangent_v"][6:10] = -0.5 * p["tangent_u"][6:10]
    return {k: v.astype(np.float32) for k, v in p.items()}


def step_gradients(scenario_index: int, step: int, seed: int = 7):
    rng = np.random.default_rng([seed, scenario_index, step])
    g = {k: rng.normal(0.0, 1.0, _shape(k, N)) * 10.0 ** rng.uniform(-4.0, 0.0, (N,) + (1,) * (WIDTH[k] > 1))
         for k in FIELDS}
    zero = rng.uniform(size=N) < 0.2
    zero[10 + step] = True
    for k in FIELDS:
        g[k][zero] = 0.0
    return {k: v.astype(np.float32) for k, v in g.items()}
