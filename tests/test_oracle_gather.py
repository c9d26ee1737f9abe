"""The oracle's gather estimator (estimator="gather") against finite
differences on the CPU: the exact derivative of the camera gather with the
photon map held, checked on a small box (300 surfels, one 32x32 camera, 16
passes) with the C3a harness (64 parameters across the seven groups,
Richardson-extrapolated central differences, eps 1e-3)."""
import numpy as np

import c3a_harness as H
from differentiablepointrendering_b200.scene import jitter_target, make_box_scene, make_surfels
from oracle_lib import OracleRenderer

ST = {"photons": 20000, "bounces": 4, "forward_passes": 1, "gather_passes": 16, "adjoint_bounces": 4,
      "adjoint_passes": 16, "gather_radius": 0.03, "gradients": "all", "rng_mode": "decorrelated",
      "estimator": "gather"}


def test_oracle_gather_estimator_matches_finite_differences():
    pts = make_surfels(300, 21)
    scene = make_box_scene(300, cameras=1, resolution=32, points=pts)
    t = OracleRenderer(scene.with_points(jitter_target(pts, 8)), ST)
    target = t.render_forward()["camera0_raw"][..., :3].astype(np.float64)
    t.close()
    r = OracleRenderer(scene, ST)
    try:
        img = r.render_forward()["camera0_raw"][..., :3].astype(np.float32)
        g, _ = r.render_backward({"camera0": ((img - target) / img.size).astype(np.float32)})
        base = r.get_point_parameters()
        params = H.draw(base, np.nonzero(np.abs(g["opacity"]) > 0)[0])

        def loss_at(p):
            r.apply_point_optimization(p)
            return H.l2_loss(r.render_gather()["camera0_raw"][..., :3], target)

        fd, fdr = H.finite_differences(loss_at, base, params)
    finally:
        r.close()
    an = np.array([H.component(g, p) for p in params])
    inp = np.array([not p[4] for p in params])
    cos, rel = H.agreement(an[inp], fdr[inp])
    assert cos >= 0.99 and rel <= 1e-2, (cos, rel)
    assert H.agreement(an[~inp], fdr[~inp])[0] >= 0.99
