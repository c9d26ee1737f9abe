"""Loads the committed GradientTests fixtures (tests/golden/gradient_tests.npz)."""
from __future__ import annotations

import os

import numpy as np

from differentiablepointrendering_b200.scene import POINT_FIELDS, SceneArrays, as_points

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "gradient_tests.npz")
KEYS = ("vertices", "triangles", "mesh_ranges", "materials", "instance_mesh", "instance_material",
        "object_to_world", "world_to_object", "camera_inv_view", "camera_forward", "camera_fovy",
        "camera_size", "camera_adjoint")


def gradient_test_scene(case: str, which: str = "initial") -> SceneArrays:
    z = np.load(PATH)
    kw = {k: z[f"{case}/{k}"] for k in KEYS}
    pts = as_points({k: z[f"{case}/{which}/{k}"] for k in POINT_FIELDS})
    return SceneArrays(**kw, camera_names=[str(s) for s in z[f"{case}/camera_names"]], points=pts)


def gradient_test_points(case: str, which: str):
    z = np.load(PATH)
    return as_points({k: z[f"{case}/{which}/{k}"] for k in POINT_FIELDS})
