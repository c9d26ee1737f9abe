"""The reference's own caller code against this renderer.

Pale's optimisation loop reaches the renderer through
python/render_hooks.py (fetch_parameters, apply_point_parameters,
rebuild_bvh, add_new_points, remove_points, get_camera_names).  This test
imports that file unchanged from the reference checkout named by
REFERENCE_CHECKOUT, with the module name `pale` bound to this package's
drop-in (differentiablepointrendering_b200.pale), and drives a small scene
through every hook.  Without the checkout it skips.
"""
import importlib.util
import os
import sys

import numpy as np
import pytest

from differentiablepointrendering_b200 import pale as drop_in
from differentiablepointrendering_b200.scene import make_box_scene

pytestmark = pytest.mark.gpu

HOOKS = os.path.join(os.environ.get("REFERENCE_CHECKOUT", ""), "python", "render_hooks.py")


@pytest.fixture(scope="module")
def hooks():
    if not os.environ.get("REFERENCE_CHECKOUT") or not os.path.exists(HOOKS):
        pytest.skip("REFERENCE_CHECKOUT does not name a reference checkout")
    saved = sys.modules.get("pale")
    sys.modules["pale"] = drop_in
    try:
        spec = importlib.util.spec_from_file_location("render_hooks_under_test", HOOKS)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        if saved is None:
            sys.modules.pop("pale", None)
        else:
            sys.modules["pale"] = saved
    return mod


def test_render_hooks_drive_the_drop_in(gpu, hooks):
    import torch

    scene = make_box_scene(2000, cameras=2, resolution=32)
    r = drop_in.Renderer.from_scene(scene, {"photons": 20000, "bounces": 3, "forward_passes": 1, "gather_passes": 1,
                                            "adjoint_bounces": 3, "adjoint_passes": 1, "gather_radius": 0.03})
    try:
        assert hooks.get_camera_names(r) == list(scene.camera_names)
        p = hooks.fetch_parameters(r)
        assert sorted(p) == sorted(["position", "tangent_u", "tangent_v", "scale", "albedo", "opacity", "beta",
                                    "shape"])
        n = p["position"].shape[0]
        assert n == 2000 and p["scale"].shape == (n, 2) and p["opacity"].shape == (n,)
        for v in p.values():
            assert v.dtype == np.float32 and v.flags["C_CONTIGUOUS"]
        # the training loop's projection hooks on torch tensors, then apply
        t = {k: torch.from_numpy(v.copy()) for k, v in p.items()}
        t["position"] += 0.001
        t["opacity"] *= 0.5
        diag = hooks.orthonormalize_tangents_inplace(t["tangent_u"], t["tangent_v"])
        assert diag["max_abs_dot_uv"] < 1e-5
        hooks.verify_scales_inplace(t["scale"])
        hooks.verify_albedos_inplace(t["albedo"])
        hooks.verify_opacities_inplace(t["opacity"])
        hooks.verify_beta_inplace(t["beta"])
        hooks.apply_point_parameters(r, t["position"], t["tangent_u"], t["tangent_v"], t["scale"], t["albedo"],
                                     t["opacity"], t["beta"])
        q = hooks.fetch_parameters(r)
        np.testing.assert_allclose(q["position"], t["position"].numpy(), rtol=0, atol=0)
        np.testing.assert_allclose(q["opacity"], t["opacity"].numpy(), rtol=0, atol=0)
        hooks.rebuild_bvh(r)
        img = r.render_forward()
        assert np.isfinite(img["camera0_raw"]).all()
        # densification: append points, then prune some by index
        k = 50
        new = {key: q[key][:k].copy() for key in ("position", "tangent_u", "tangent_v", "scale", "albedo", "opacity",
                                                   "beta")}
        new["position"] = new["position"] + 0.002
        hooks.add_new_points(r, {"new": new})
        hooks.add_new_points(r, None)
        assert hooks.fetch_parameters(r)["position"].shape[0] == n + k
        hooks.remove_points(r, np.arange(0, n + k, 7))
        left = n + k - len(range(0, n + k, 7))
        q2 = hooks.fetch_parameters(r)
        assert q2["position"].shape[0] == left
        hooks.rebuild_bvh(r)
        img2 = r.render_forward()
        raw = img2["camera0_raw"][..., :3]
        grads, _ = r.render_backward({"camera0": (raw / raw.size).astype(np.float32)})
        assert grads["opacity"].shape == (left,)
        with pytest.raises(ValueError):
            hooks.remove_points(r, np.zeros((2, 2), np.int64))
    finally:
        r.close()
