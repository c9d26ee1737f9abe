"""The serving loop (serving.Server) on the GPU: resident scenes with
their photon maps traced once, requests of several scenes, passes and
depths batched into rounds (one camera-gather wavefront per round, and for
the gradient requests a shared adjoint wavefront of the reference's
adjoint or a sweep of the gather estimator over the round's own path
vertices), and every result the same alone and in the mix: images and
losses bit for bit, gradients up to the order of float atomic additions."""
import threading

import numpy as np
import pytest

from differentiablepointrendering_b200.scene import POINT_FIELDS, make_box_scene, make_surfels

pytestmark = pytest.mark.gpu

SETTINGS = {"photons": 20000, "bounces": 3, "forward_passes": 1, "gather_passes": 4, "adjoint_bounces": 4,
            "adjoint_passes": 4, "gather_radius": 0.03}


def _scenes():
    a = make_box_scene(3000, cameras=2, resolutions=[32, 48], points=make_surfels(3000, 5))
    b = make_box_scene(6000, cameras=3, resolution=64, points=make_surfels(6000, 9))
    return a, b


@pytest.mark.parametrize("estimator", ["reference", "gather"])
def test_results_are_the_same_alone_and_in_the_mix(gpu, estimator):
    import torch

    from differentiablepointrendering_b200.serving import Request, Server

    free, _ = torch.cuda.mem_get_info()
    # the gather variant computes every gradient group, the reference one opacity only
    groups = "all" if estimator == "gather" else "opacity"
    srv = Server(hbm_budget=free, settings={"rng_mode": "decorrelated", "estimator": estimator,
                                            "gradients": groups})
    try:
        a, b = _scenes()
        srv.add_scene("a", a, SETTINGS)
        srv.add_scene("b", b, SETTINGS)
        sizes = {"a": a.camera_size, "b": b.camera_size}
        # the planner's per-view cost: surfel layers per camera path, measured at admission
        for name, sc in (("a", a), ("b", b)):
            assert len(srv.scenes[name].layers) == len(sc.camera_size)
            assert all(x > 0 for x in srv.scenes[name].layers)
        rng = np.random.default_rng(4)
        specs = []
        for _ in range(32):
            s = "a" if rng.uniform() < 0.5 else "b"
            cam = int(rng.integers(len(sizes[s])))
            w, h = (int(x) for x in sizes[s][cam])
            passes, depth = int(rng.integers(1, 5)), int(rng.integers(0, 5))
            if rng.uniform() < 0.4:
                specs.append((s, cam, "gradient", rng.uniform(0, 1, (h, w, 3)).astype(np.float32), passes, depth))
            else:
                specs.append((s, cam, "forward", None, passes, depth))
        mix = [Request(s, c, k, t, p, d) for s, c, k, t, p, d in specs]
        # submitted from four threads at once
        parts = [mix[i::4] for i in range(4)]
        threads = [threading.Thread(target=lambda p=p: [srv.submit(q) for q in p]) for p in parts]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for q in mix:
            assert q.done.wait(120), q
            assert q.error is None, q.error
        assert max(q.batch_views for q in mix) > 1                 # some requests shared a round
        assert sum(1 for q in mix if q.kind == "gradient") >= 2
        lit = 0
        for q in mix:
            alone = srv.serve_one(Request(q.scene, q.camera, q.kind, q.target, q.passes, q.depth))
            assert alone.error is None, alone.error
            assert alone.batch_views == 1
            np.testing.assert_array_equal(alone.image, q.image)
            if q.kind == "gradient":
                assert alone.loss == q.loss
                # only the computed groups come back
                assert set(q.grads) == ({"opacity"} if groups == "opacity" else set(POINT_FIELDS))
                for key in ("opacity", "albedo") if estimator == "gather" else ("opacity",):
                    a_, b_ = alone.grads[key].astype(np.float64), q.grads[key].astype(np.float64)
                    # a camera that looks at a closed wall of the box from outside sees no surfel
                    assert np.linalg.norm(a_ - b_) <= 1e-4 * np.linalg.norm(b_), (key, q)
                    lit += int(np.linalg.norm(b_) > 0)
        assert lit >= 2
        lat = srv.latency()
        assert lat["n"] >= len(mix) and lat["p99"] >= lat["p50"] > 0
    finally:
        srv.close()


def test_admission_refuses_scenes_beyond_the_budget(gpu):
    from differentiablepointrendering_b200.serving import AdmissionError, Server

    srv = Server(hbm_budget=1)
    try:
        a, _ = _scenes()
        with pytest.raises(AdmissionError):
            srv.add_scene("a", a, SETTINGS)
        assert not srv.scenes
    finally:
        srv.close()


@pytest.mark.parametrize("policy", ["arrival", "light_first"])
def test_forward_requests_in_slices_equal_alone(gpu, policy):
    """With a round cap of 4096 camera paths, a 64x64 request of 4 passes
    renders in slices over several rounds (its running sums carried between
    them) while other requests get rounds in between: its image is bit for
    bit the one of the request rendered in one call."""
    import torch

    from differentiablepointrendering_b200.serving import Request, Server

    free, _ = torch.cuda.mem_get_info()
    srv = Server(hbm_budget=free, settings={"rng_mode": "decorrelated"}, max_paths=4096, policy=policy)
    try:
        a, b = _scenes()
        srv.add_scene("a", a, SETTINGS)
        srv.add_scene("b", b, SETTINGS)
        mix = [Request("b", k % 3, "forward", None, 4, 0) for k in range(6)] + \
              [Request("a", k % 4, "forward", None, 1 + k % 4, 0) for k in range(6)]
        for q in mix:
            srv.submit(q)
        for q in mix:
            assert q.done.wait(120), q
            assert q.error is None, q.error
        assert max(q.slices for q in mix) > 1
        for q in mix:
            alone = srv.serve_one(Request(q.scene, q.camera, q.kind, None, q.passes, q.depth))
            assert alone.error is None and alone.slices == 1
            np.testing.assert_array_equal(alone.image, q.image)
    finally:
        srv.close()


def test_gradient_requests_in_slices_equal_alone(gpu):
    """With a round cap of 4096 camera paths, 64x64 gradient requests of 4
    passes render their forward in slices over several rounds and their
    adjoint in the round of the last slice: image and loss bit for bit those
    of the request alone, gradients up to the order of float atomic
    additions."""
    import torch

    from differentiablepointrendering_b200.serving import Request, Server

    free, _ = torch.cuda.mem_get_info()
    srv = Server(hbm_budget=free, settings={"rng_mode": "decorrelated"}, max_paths=4096, policy="light_first")
    try:
        a, b = _scenes()
        srv.add_scene("a", a, SETTINGS)
        srv.add_scene("b", b, SETTINGS)
        rng = np.random.default_rng(6)
        mix = [Request("b", k % 3, "gradient", rng.uniform(0, 1, (64, 64, 3)).astype(np.float32), 4, 2)
               for k in range(4)] + [Request("a", k % 4, "forward", None, 1 + k % 4, 0) for k in range(6)]
        for q in mix:
            srv.submit(q)
        for q in mix:
            assert q.done.wait(120), q
            assert q.error is None, q.error
        grads = [q for q in mix if q.kind == "gradient"]
        assert max(q.slices for q in grads) > 1
        lit = 0
        for q in grads:
            alone = srv.serve_one(Request(q.scene, q.camera, q.kind, q.target, q.passes, q.depth))
            assert alone.error is None and alone.slices == 1
            np.testing.assert_array_equal(alone.image, q.image)
            assert alone.loss == q.loss
            a_, b_ = alone.grads["opacity"].astype(np.float64), q.grads["opacity"].astype(np.float64)
            assert np.linalg.norm(a_ - b_) <= 1e-4 * np.linalg.norm(b_)
            lit += int(np.linalg.norm(b_) > 0)
        assert lit >= 1
    finally:
        srv.close()
