"""Generates tests/golden/gradient_tests.npz from Pale's GradientTests scenes.

Run in a container that has the reference checkout:

    python tests/golden/make_fixtures.py /path/to/DifferentiablePointRendering

It parses Assets/GradientTests/<case>/<case>.xml with initial.ply and
target.ply (the scenes of python/finite_difference/tests.json and their
siblings) through this package's Mitsuba/PLY readers and stores the
resulting arrays, so the tests need no reference checkout at run time.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from differentiablepointrendering_b200.scene import (POINT_FIELDS, load_mitsuba_scene,  # noqa: E402
                                                     load_surfel_ply)

CASES = ("empty", "simple_1", "simple_2", "simple_3", "scatter", "transmit")
SCENE_KEYS = ("vertices", "triangles", "mesh_ranges", "materials", "instance_mesh", "instance_material",
              "object_to_world", "world_to_object", "camera_inv_view", "camera_forward", "camera_fovy",
              "camera_size", "camera_adjoint")


def main(ref_root: str):
    assets = os.path.join(ref_root, "Assets")
    out = {}
    for case in CASES:
        d = os.path.join(assets, "GradientTests", case)
        init = load_surfel_ply(os.path.join(d, "initial.ply"))
        tgt = load_surfel_ply(os.path.join(d, "target.ply"))
        sc = load_mitsuba_scene(assets, os.path.join(d, f"{case}.xml"), init)
        for k in SCENE_KEYS:
            out[f"{case}/{k}"] = np.asarray(getattr(sc, k))
        out[f"{case}/camera_names"] = np.asarray(sc.camera_names)
        for k in POINT_FIELDS:
            out[f"{case}/initial/{k}"] = init[k]
            out[f"{case}/target/{k}"] = tgt[k]
    path = os.path.join(HERE, "gradient_tests.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the reference checkout>")
    main(sys.argv[1])
