"""The reference's own gradient check (fd_harness) on the CUDA renderer.

1. fd_test.py's settings (1e6 photons x 50 forward passes, 5 bounces,
   1 gather pass, 1 adjoint bounce, 8 adjoint passes, seed 42) at the
   scenes' 500x500, through the drop-in Renderer surface:
   set_point_opacity(opacity, index) and rebuild_bvh() before every render.
   `empty` passes.  `simple_1` does not, and cannot with the reference's
   algorithm, which this renderer and the oracle restate identically.  Its
   surfel sits 0.2 in front of a lit wall.  The finite difference retraces
   the photons, so it also sees the opacity change the photon map (the
   surfel shadows the wall), which the adjoint does not follow; with one
   adjoint bounce a NullTransmittance (occlusion) event never completes,
   as its endpoint is the next hit; and when it does, the reference weights
   it by qNull too little.  The test records that as an expected failure
   (strict: it is reported if it ever passes).
2. The same sweep with the photon map held at the base value's
   (render_gather), 2 adjoint bounces, decorrelated adjoint passes and the
   unbiased NullTransmittance weight (null_weight "unbiased": the reference
   weights those events by qNull too little): what the adjoint
   differentiates.  Both scenes pass the reference's thresholds.
3. render_gather right after render_forward returns the same images.
"""
import numpy as np
import pytest

import fd_harness as H
from differentiablepointrendering_b200.pale import Renderer

pytestmark = pytest.mark.gpu

SETTINGS = {"photons": 1e6, "bounces": 5, "forward_passes": 50, "gather_passes": 1, "adjoint_bounces": 1,
            "adjoint_passes": 8, "logging": 4, "seed": 42}
FROZEN = dict(SETTINGS, adjoint_bounces=2, adjoint_passes=32, rng_mode="decorrelated", null_weight="unbiased")


def _set_opacity(r, value):
    r.set_point_opacity(opacity=float(value), index=0)
    r.rebuild_bvh()


def _run(case, settings):
    t = Renderer.from_scene(H.scene(case, "target"), settings)
    target = H.raw_rgb(t)
    t.close()
    r = Renderer.from_scene(H.scene(case, "initial"), settings)
    try:
        return H.sweep(r, target, _set_opacity)
    finally:
        r.close()


def test_fd_check_empty(gpu):
    rows = _run("empty", SETTINGS)
    assert not H.failing_rows(rows), (H.failing_rows(rows), rows)
    assert max(abs(fd) for _, _, fd in rows) > 1e-3


@pytest.mark.xfail(strict=True, reason="the reference's adjoint does not follow the photon map and, with one "
                                       "adjoint bounce, drops the occlusion term; its FD harness sees both")
def test_fd_check_simple_1(gpu):
    rows = _run("simple_1", SETTINGS)
    assert not H.failing_rows(rows), (H.failing_rows(rows), rows)


def _frozen_sweep(case):
    """fd_harness.sweep with the finite difference taken by render_gather
    on the photon map traced at the base value."""
    t = Renderer.from_scene(H.scene(case, "target"), FROZEN)
    target = H.raw_rgb(t)
    t.close()
    r = Renderer.from_scene(H.scene(case, "initial"), FROZEN)

    def gathered():
        return np.asarray(r.render_gather()[H.CAMERA + "_raw"], np.float32)[..., :3]

    rows = []
    try:
        for it in range(H.ITERATIONS + 1):
            v = it / H.ITERATIONS
            _set_opacity(r, v)
            base = H.raw_rgb(r)              # traces the photon map at v
            lo, hi = max(0.0, v - H.EPS), min(1.0, v + H.EPS)
            _set_opacity(r, hi)
            lp = H.l2_loss(gathered(), target)
            _set_opacity(r, lo)
            lm = H.l2_loss(gathered(), target)
            _set_opacity(r, v)
            grads, _ = r.render_backward({H.CAMERA: ((base - target) / base.size).astype(np.float32)})
            rows.append((v, float(grads["opacity"][0]), (lp - lm) / (hi - lo)))
    finally:
        r.close()
    return rows


@pytest.mark.parametrize("case", ["empty", "simple_1"])
def test_fd_check_with_photon_map_held(gpu, case):
    rows = _frozen_sweep(case)
    assert not H.failing_rows(rows), (H.failing_rows(rows), rows)


def test_render_gather_reproduces_forward(gpu):
    r = Renderer.from_scene(H.scene("simple_1", "initial", 96), SETTINGS)
    try:
        a = r.render_forward()
        b = r.render_gather()
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])
    finally:
        r.close()


# ---------------------------------------------------------------- a23 groups
GROUPS = dict(FROZEN, gather_passes=16, adjoint_passes=64, gradients="all")
# parameters whose effect on the image goes through the surfel's alpha_geom
# (and albedo): the in-plane tangent/position components, scale, beta,
# albedo, opacity.  Moving the surfel out of its plane also moves its hit
# points against the photons deposited on it (E(x) changes), which the
# reference's derivative formulas do not model.
ALPHA_DRIVEN = [("opacity", 0, 5e-3), ("beta", 0, 1e-2), ("albedo", 0, 1e-2), ("albedo", 1, 1e-2),
                ("albedo", 2, 1e-2), ("scale", 0, 2e-4), ("scale", 1, 2e-4), ("tangent_u", 0, 2e-3),
                ("tangent_v", 2, 2e-3), ("position", 2, 2e-4)]


def test_all_gradient_groups_match_finite_differences(gpu):
    """Every group's gradient of the one surfel of `simple_1` (opacity set to
    0.6) against a central difference of the loss with the photon map held
    (render_gather); 16 gather passes so that the forward image is close to
    the pixel integral the adjoint estimates."""
    t = Renderer.from_scene(H.scene("simple_1", "target"), GROUPS)
    target = H.raw_rgb(t)
    t.close()
    r = Renderer.from_scene(H.scene("simple_1", "initial"), GROUPS)
    try:
        base = r.get_point_parameters()
        base["opacity"][0] = 0.6
        r.apply_point_optimization(base)
        img = H.raw_rgb(r)
        grads, _ = r.render_backward({H.CAMERA: ((img - target) / img.size).astype(np.float32)})

        def loss(params):
            r.apply_point_optimization(params)
            return H.l2_loss(np.asarray(r.render_gather()[H.CAMERA + "_raw"], np.float32)[..., :3], target)

        rows = []
        for key, comp, eps in ALPHA_DRIVEN:
            shape = base[key].reshape(len(base[key]), -1).shape
            vals = []
            for sgn in (1, -1):
                p = {k: v.copy() for k, v in base.items()}
                p[key].reshape(shape)[0, comp] += sgn * eps
                vals.append(loss(p))
            fd = (vals[0] - vals[1]) / (2 * eps)
            an = float(np.asarray(grads[key]).reshape(shape)[0, comp])
            rows.append((key, comp, an, fd))
        r.apply_point_optimization(base)
    finally:
        r.close()
    scale = max(abs(fd) for *_, fd in rows)
    bad = [(k, c, an, fd) for k, c, an, fd in rows
           if abs(an - fd) / max(1e-30, abs(an) + abs(fd)) > 0.1 and abs(an - fd) > 0.02 * scale]
    assert not bad, (bad, rows)
