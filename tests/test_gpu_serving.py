"""The serving loop (serving.Server): resident scenes on per-scene streams,
forward requests merged into shared calls, and results that are the same
alone and in the mix."""
import threading

import numpy as np
import pytest

from differentiablepointrendering_b200.scene import make_box_scene, make_surfels

pytestmark = pytest.mark.gpu

SETTINGS = {"photons": 20000, "bounces": 3, "forward_passes": 1, "gather_passes": 2, "adjoint_bounces": 3,
            "adjoint_passes": 2, "gather_radius": 0.03}


def _scenes():
    a = make_box_scene(3000, cameras=4, resolution=48, points=make_surfels(3000, 5))
    b = make_box_scene(6000, cameras=3, resolution=64, points=make_surfels(6000, 9))
    return a, b


def test_results_are_the_same_alone_and_in_the_mix(gpu):
    import torch

    from differentiablepointrendering_b200.serving import Request, Server

    free, _ = torch.cuda.mem_get_info()
    srv = Server(hbm_budget=free)
    try:
        a, b = _scenes()
        srv.add_scene("a", a, SETTINGS)
        srv.add_scene("b", b, SETTINGS)
        rng = np.random.default_rng(4)
        specs = []
        for _ in range(24):
            s = "a" if rng.uniform() < 0.5 else "b"
            cams, res = (4, 48) if s == "a" else (3, 64)
            cam = int(rng.integers(cams))
            if rng.uniform() < 0.25:
                specs.append((s, cam, "gradient", rng.uniform(0, 1, (res, res, 3)).astype(np.float32)))
            else:
                specs.append((s, cam, "forward", None))
        mix = [Request(s, c, k, t) for s, c, k, t in specs]
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
        assert max(q.batch_views for q in mix if q.kind == "forward") > 1   # some forwards shared a call
        for q in mix:
            alone = srv.submit(Request(q.scene, q.camera, q.kind, q.target))
            assert alone.done.wait(120) and alone.error is None
            assert alone.batch_views == 1
            np.testing.assert_array_equal(alone.image, q.image)
            if q.kind == "gradient":
                assert alone.loss == q.loss
                for k, v in alone.grads.items():
                    scale = float(np.abs(v).max()) + 1e-30
                    np.testing.assert_allclose(q.grads[k], v, rtol=1e-4, atol=1e-6 * scale, err_msg=k)
        lat = srv.latency()
        assert lat["n"] == 2 * len(mix) and lat["p99"] >= lat["p50"] > 0
    finally:
        srv.close()


def test_admission_by_hbm_budget(gpu):
    from differentiablepointrendering_b200.serving import AdmissionError, Server

    a, b = _scenes()
    srv = Server(hbm_budget=1 << 20)
    try:
        with pytest.raises(AdmissionError):
            srv.add_scene("a", a, SETTINGS)
        assert not srv.scenes
    finally:
        srv.close()
    big = Server(hbm_budget=1 << 40)
    try:
        need = big.add_scene("a", a, SETTINGS)
        assert need > 0
    finally:
        big.close()
    one = Server(hbm_budget=need + need // 2)
    try:
        one.add_scene("a", a, SETTINGS)
        with pytest.raises(AdmissionError):
            one.add_scene("b", b, SETTINGS)
        assert list(one.scenes) == ["a"]
    finally:
        one.close()
