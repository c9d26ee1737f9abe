"""The gather estimator (estimator="gather"): the exact derivative of the
camera gather's image with the photon map held, on the forward's own camera
paths, swept from checkpointed path vertices or from chunks traced again by
deterministic replay.

C3a: 1k surfels in the box, one 64x64 camera, 256 passes, 100k photons,
radius 0.02, all seven gradient groups.  The CUDA gradient against the
oracle's restatement of the same derivative (all groups, cosine >= 0.99
and relative L2 <= 1e-2), and against central finite differences of the
loss on 64 parameters drawn with seed 99 across the seven groups (the
c3a_harness module: eps 1e-3 with Richardson's extrapolation; cosine
>= 0.99 and relative L2 <= 1e-2 over the parameters that move a surfel
within its plane, the out-of-plane ones at cosine >= 0.99 and reported).
Checkpoint, replay and a store that holds only some chunks give the same
gradients up to the order of float atomic additions."""
import numpy as np
import pytest

import c3a_harness as H
from differentiablepointrendering_b200.pale import Renderer
from differentiablepointrendering_b200.scene import jitter_target, make_box_scene, make_surfels
from oracle_lib import OracleRenderer

pytestmark = pytest.mark.gpu

C3A = {"photons": 100000, "bounces": 4, "forward_passes": 1, "gather_passes": 256, "adjoint_bounces": 4,
       "adjoint_passes": 256, "gather_radius": 0.02, "gradients": "all", "rng_mode": "decorrelated",
       "estimator": "gather"}
GROUP_KEYS = ("opacity", "beta", "albedo", "scale", "position", "tangent_u", "tangent_v")


@pytest.fixture(scope="module")
def c3a():
    pts = make_surfels(1000, 1234)
    scene = make_box_scene(1000, cameras=1, resolution=64, points=pts)
    return scene, scene.with_points(jitter_target(pts, 5678))


def _raw(images, cam="camera0"):
    return np.asarray(images[cam + "_raw"], np.float32)[..., :3]


def _dl(img, target):
    return ((img - target) / img.size).astype(np.float32)


def _to_asset(values, order):
    out = np.empty_like(values)
    out[order] = values
    return out


def test_gather_estimator_matches_the_oracle(gpu, c3a):
    scene, tscene = c3a
    t = OracleRenderer(tscene, C3A)
    target = _raw(t.render_forward())
    t.close()
    g = Renderer.from_scene(scene, C3A)
    o = OracleRenderer(scene, C3A)
    try:
        ig, io = _raw(g.render_forward()), _raw(o.render_forward())
        gg, _ = g.render_backward({"camera0": _dl(ig, target)})
        go, _ = o.render_backward({"camera0": _dl(io, target)})
        og, oo = g.get_point_order(), o.get_point_order()
        for k in GROUP_KEYS:
            a, b = _to_asset(gg[k], og), _to_asset(go[k], oo)
            assert np.linalg.norm(b) > 0, k
            cos, rel = H.agreement(a.reshape(-1), b.reshape(-1))
            assert cos >= 0.99 and rel <= 1e-2, (k, cos, rel)
    finally:
        g.close()
        o.close()


def _grads(r, target, cams=None):
    img = r.render_forward()
    dl = {c: _dl(_raw(img, c), _raw(target, c)) for c in (cams or r.get_camera_names())}
    g, _ = r.render_backward(dl)
    return g, r.stats()


def test_checkpoint_replay_and_partial_store_agree(gpu):
    """Two cameras, 16 passes in chunks of one pass of both cameras: the
    replay gradient against a full checkpoint (the store grown by a first
    iteration) and against a store sized by a forward of one camera, which
    holds about half of the chunks and replays the rest."""
    pts = make_surfels(3000, 77)
    scene = make_box_scene(3000, cameras=2, resolution=48, points=pts)
    st = dict(C3A, gather_passes=16, adjoint_passes=16, gather_batch_paths=2 * 48 * 48)
    t = Renderer.from_scene(scene.with_points(jitter_target(pts, 5)), st)
    target = t.render_forward()
    t.close()
    runs = {}
    for mode in ("replay", "checkpoint", "partial"):
        r = Renderer.from_scene(scene, dict(st, vertices="replay" if mode == "replay" else "checkpoint"))
        try:
            if mode == "checkpoint":
                _grads(r, target)                    # grows the store
            if mode == "partial":
                r.render_forward("camera0")          # a store for one camera's chunks
                r.render_backward({"camera0": _dl(_raw(target, "camera0"), _raw(target, "camera0"))})
            runs[mode] = _grads(r, target)
        finally:
            r.close()
    assert runs["replay"][1]["vertex_chunks_stored"] == 0 and runs["replay"][1]["vertex_chunks_replayed"] == 16
    assert runs["checkpoint"][1]["vertex_chunks_stored"] == 16
    sp, rp = runs["partial"][1]["vertex_chunks_stored"], runs["partial"][1]["vertex_chunks_replayed"]
    assert sp > 0 and rp > 0 and sp + rp == 16, (sp, rp)
    for mode in ("checkpoint", "partial"):
        for k in GROUP_KEYS:
            a, b = runs[mode][0][k].reshape(-1), runs["replay"][0][k].reshape(-1)
            assert np.linalg.norm(b) > 0, k
            cos, rel = H.agreement(a, b)
            assert cos >= 0.99999 and rel <= 1e-4, (mode, k, cos, rel)


def test_c3a_finite_differences(gpu, c3a):
    scene, tscene = c3a
    t = Renderer.from_scene(tscene, C3A)
    target = _raw(t.render_forward()).astype(np.float64)
    t.close()
    r = Renderer.from_scene(scene, C3A)
    try:
        img = _raw(r.render_forward())
        g, _ = r.render_backward({"camera0": _dl(img, target.astype(np.float32))})
        base = r.get_point_parameters()
        params = H.draw(base, np.nonzero(np.abs(g["opacity"]) > 0)[0])

        def loss_at(p):
            r.apply_point_optimization(p)
            return H.l2_loss(_raw(r.render_gather()), target)

        fd, fdr = H.finite_differences(loss_at, base, params)
    finally:
        r.close()
    an = np.array([H.component(g, p) for p in params])
    inp = np.array([not p[4] for p in params])
    assert {p[0] for p in params} == set(GROUP_KEYS) and inp.sum() >= 40
    cos, rel = H.agreement(an[inp], fdr[inp])
    assert cos >= 0.99 and rel <= 1e-2, (cos, rel, H.agreement(an[inp], fd[inp]))
    cos_o, rel_o = H.agreement(an[~inp], fdr[~inp])
    assert cos_o >= 0.99, (cos_o, rel_o)


def test_backward_needs_the_forward_it_differentiates(gpu):
    scene = make_box_scene(500, cameras=1, resolution=32)
    r = Renderer.from_scene(scene, dict(C3A, gather_passes=2, adjoint_passes=2))
    try:
        img = _raw(r.render_forward())
        p = r.get_point_parameters()
        r.apply_point_optimization(p)                # the points changed since the forward
        with pytest.raises(RuntimeError, match="last forward render"):
            r.render_backward({"camera0": np.zeros_like(img)})
        r.render_forward()
        g, _ = r.render_backward({"camera0": np.ones_like(img) * 1e-3})
        assert np.isfinite(g["opacity"]).all()
    finally:
        r.close()
