"""The serving loop's host logic on CPU, with a stand-in renderer: a worker
merges the queued forward requests of its scene into calls over at most
max_views sorted cameras and then runs the gradient requests one at a time
in arrival order; submit validates requests; add_scene admits scenes by
their measured footprint against the HBM budget and forces camera-keyed
seeds."""
import threading

import numpy as np
import pytest

import differentiablepointrendering_b200.serving as S


class FakeRenderer:
    def __init__(self, ncams=6, size=(4, 3)):
        self._names = [f"cam{i}" for i in range(ncams)]
        self._sizes = [size] * ncams
        self.closed = False
        self.settings = None

    def get_camera_names(self):
        return list(self._names)

    def render_forward(self):
        return {}

    def render_backward(self, d):
        return {}, {}

    def close(self):
        self.closed = True


class RecordingScene(S._Scene):
    """A worker whose device calls only record what they were given."""

    def __init__(self, *a, **k):
        super().__init__(*a, **k)
        self.calls = []

    def _forward(self, cams, reqs):
        self.calls.append(("forward", list(cams), sorted(q.camera for q in reqs)))
        for q in reqs:
            q.batch_views = len(cams)
            self._finish(q)

    def _gradient(self, q):
        self.calls.append(("gradient", q.camera))
        self._finish(q)


def test_worker_merges_forwards_then_runs_gradients_in_order():
    sc = RecordingScene("s", FakeRenderer(), footprint=0, max_views=2)
    reqs = [S.Request("s", c) for c in (3, 1, 3, 2, 5)]
    grads = [S.Request("s", c, kind="gradient", target=np.zeros((3, 4, 3), np.float32)) for c in (4, 0)]
    # queue everything before the worker starts, so that it takes one batch
    sc.queue = reqs[:2] + [grads[0]] + reqs[2:] + [grads[1]]
    sc.thread.start()
    for q in reqs + grads:
        assert q.done.wait(10)
    with sc.cv:
        sc.stop = True
        sc.cv.notify()
    sc.thread.join(10)
    assert sc.calls == [("forward", [1, 2], [1, 2]), ("forward", [3, 5], [3, 3, 5]),
                        ("gradient", 4), ("gradient", 0)]
    assert [q.batch_views for q in reqs] == [2, 2, 2, 2, 2]
    assert all(q.latency_ms >= 0 for q in reqs)


def _server_with_fake_scene():
    srv = S.Server(hbm_budget=1 << 30)
    sc = RecordingScene("s", FakeRenderer(), footprint=0, max_views=4)
    srv.scenes["s"] = sc
    sc.thread.start()
    return srv, sc


def test_submit_validates_and_latency_reports():
    srv, sc = _server_with_fake_scene()
    try:
        with pytest.raises(KeyError):
            srv.submit(S.Request("nope", 0))
        with pytest.raises(ValueError):
            srv.submit(S.Request("s", 0, kind="backward"))
        with pytest.raises(IndexError):
            srv.submit(S.Request("s", 6))
        with pytest.raises(ValueError):
            srv.submit(S.Request("s", 0, kind="gradient"))
        assert srv.latency() == {"n": 0}
        qs = [srv.submit(S.Request("s", c)) for c in (0, 1, 2)]
        for q in qs:
            assert q.done.wait(10)
        lat = srv.latency("forward")
        assert lat["n"] == 3 and 0 <= lat["p50"] <= lat["p99"]
        assert srv.latency("gradient") == {"n": 0}
    finally:
        srv.close()
    assert sc.r.closed


def test_admission_by_measured_footprint(monkeypatch):
    made = []

    def from_scene(scene, settings):
        r = FakeRenderer()
        r.settings = settings
        made.append(r)
        return r

    used = {"v": 0}
    lock = threading.Lock()

    def device_used():
        with lock:
            return used["v"]

    def forward(self):
        used["v"] += 6 << 30       # every renderer holds 6 GiB after its first passes
        return {}

    monkeypatch.setattr(S.Renderer, "from_scene", staticmethod(from_scene))
    monkeypatch.setattr(S, "_device_used", device_used)
    monkeypatch.setattr(FakeRenderer, "render_forward", forward)
    srv = S.Server(hbm_budget=10 << 30)
    try:
        assert srv.add_scene("a", scene=None, settings={"photons": 10}) == 6 << 30
        assert made[0].settings == {"photons": 10, "camera_seeds": "camera"}
        with pytest.raises(ValueError):
            srv.add_scene("a", scene=None)
        with pytest.raises(S.AdmissionError):
            srv.add_scene("b", scene=None)
        assert made[1].closed and "b" not in srv.scenes
        assert srv.admitted_bytes == 6 << 30
    finally:
        srv.close()
    assert made[0].closed
