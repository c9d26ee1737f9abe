"""The serving loop's host logic on CPU: how a round is planned from the
queue (arrival order, view and pixel caps, the first request always goes)
and how submit validates requests against the resident scene (camera,
passes and depth ranges, gradient targets)."""
import threading

import numpy as np
import pytest

import differentiablepointrendering_b200.serving as S


def _sizes():
    return {"a": [(4, 4), (8, 8)], "b": [(16, 16)]}


def test_round_takes_the_queue_head_in_arrival_order():
    q = [S.Request("a", 0), S.Request("b", 0), S.Request("a", 1), S.Request("a", 0)]
    taken, left = S.plan_round(q, _sizes(), max_views=3, max_pixels=10 ** 6)
    assert taken == q[:3] and left == q[3:]
    taken, left = S.plan_round(q, _sizes(), max_views=64, max_pixels=10 ** 6)
    assert taken == q and left == []


def test_round_respects_the_pixel_cap_but_always_takes_one():
    q = [S.Request("b", 0), S.Request("a", 0), S.Request("a", 1)]
    taken, left = S.plan_round(q, _sizes(), max_views=64, max_pixels=100)
    assert taken == q[:1] and left == q[1:]          # 256 pixels > cap: alone
    taken, left = S.plan_round(q[1:], _sizes(), max_views=64, max_pixels=80)
    assert taken == q[1:3] and left == []            # 16 + 64 = 80
    taken, left = S.plan_round(q[1:], _sizes(), max_views=64, max_pixels=79)
    assert taken == q[1:2] and left == q[2:]


class _FakeRenderer:
    _names = ["c0", "c1"]
    _sizes = [(4, 3), (4, 3)]


def _server():
    srv = S.Server.__new__(S.Server)     # host logic only: no executor, no thread
    srv.scenes = {"s": S._Scene("s", _FakeRenderer(), 0, max_passes=16, max_depth=6)}
    srv.done, srv._queue = [], []
    srv._cv, srv._lock = threading.Condition(), threading.Lock()
    return srv


def test_submit_validates_requests():
    srv = _server()
    with pytest.raises(KeyError):
        srv.submit(S.Request("nope", 0))
    with pytest.raises(ValueError):
        srv.submit(S.Request("s", 0, kind="backward"))
    with pytest.raises(IndexError):
        srv.submit(S.Request("s", 2))
    with pytest.raises(ValueError):
        srv.submit(S.Request("s", 0, kind="gradient"))
    with pytest.raises(ValueError):
        srv.submit(S.Request("s", 0, passes=17))
    with pytest.raises(ValueError):
        srv.submit(S.Request("s", 0, depth=7))
    q = srv.submit(S.Request("s", 1, kind="gradient", target=np.zeros((3, 4, 3), np.float32), passes=4, depth=2))
    assert srv._queue == [q] and q.t_submit > 0


def test_round_respects_the_path_cap():
    q = [S.Request("a", 1, passes=4), S.Request("a", 1), S.Request("b", 0, passes=1)]
    spp = {"a": 8, "b": 8}
    # 64*4 = 256 paths, then 64*8 = 512 (passes 0: the scene's maximum), then 256*1 = 256
    taken, left = S.plan_round(q, _sizes(), 64, 10 ** 6, max_paths=1023, max_passes=spp)
    assert taken == q[:2] and left == q[2:]
    taken, left = S.plan_round(q, _sizes(), 64, 10 ** 6, max_paths=1024, max_passes=spp)
    assert taken == q and left == []
    taken, left = S.plan_round(q, _sizes(), 64, 10 ** 6, max_paths=10, max_passes=spp)
    assert taken == q[:1]


def test_round_holds_at_most_seven_scenes():
    sizes = {f"s{k}": [(4, 4)] for k in range(9)}
    q = [S.Request(f"s{k}", 0) for k in range(9)] + [S.Request("s0", 0)]
    taken, left = S.plan_round(q, sizes, 64, 10 ** 6)
    assert [r.scene for r in taken] == [f"s{k}" for k in range(7)] and left == q[7:]
    taken, left = S.plan_round(q, sizes, 64, 10 ** 6, max_scenes=2)
    assert taken == q[:2]


def test_light_first_takes_light_requests_past_a_heavy_one():
    sizes = {"a": [(4, 4), (64, 64)]}
    heavy = S.Request("a", 1, passes=8)                  # 32768 paths
    light = [S.Request("a", 0, passes=1) for _ in range(3)]
    grad = S.Request("a", 0, kind="gradient", passes=1)  # 16 paths, counted twice
    for k, q in enumerate([heavy] + light + [grad]):
        q.t_submit = 10.0 + k * 0.01
    q = [heavy] + light + [grad]
    taken, left = S.plan_round(q, sizes, 64, 10 ** 6, max_paths=1000, policy="light_first", now=10.5)
    assert taken == light + [grad] and left == [heavy]
    # the arrival order stops at the heavy head
    taken, left = S.plan_round(q, sizes, 64, 10 ** 6, max_paths=1000, now=10.5)
    assert taken == [heavy] and left == light + [grad]
    # a request that waited past starve_s goes first
    taken, left = S.plan_round(q, sizes, 64, 10 ** 6, max_paths=1000, policy="light_first", now=13.0,
                               starve_s=2.0)
    assert taken == [heavy] and left == light + [grad]


def test_light_first_round_stays_light():
    sizes = {"a": [(4, 4), (1024, 1024)]}
    light = S.Request("a", 0, passes=1)                   # 16 paths
    medium = S.Request("a", 1, passes=2)                  # 2M paths
    for k, q in enumerate([light, medium]):
        q.t_submit = 1.0 + 0.01 * k
    taken, left = S.plan_round([light, medium], sizes, 64, 1 << 24, max_paths=1 << 24,
                               policy="light_first", now=1.1)
    assert taken == [light] and left == [medium]         # 2M > max(2^20, 8 x 16)
    taken, left = S.plan_round([medium], sizes, 64, 1 << 24, max_paths=1 << 24, policy="light_first", now=1.1)
    assert taken == [medium]


def test_light_first_weighs_paths_by_the_views_layers():
    # two views of one size: camera 0 sees a wall (1 layer per path),
    # camera 1 looks into a dense cloud (150 layers per path)
    sizes = {"a": [(512, 512), (512, 512)]}
    layers = {"a": [1.0, 150.0]}
    dense = S.Request("a", 1, kind="gradient", passes=1)
    walls = [S.Request("a", 0, kind="gradient", passes=1) for _ in range(3)]
    for k, q in enumerate([dense] + walls):
        q.t_submit = 1.0 + 0.01 * k
    q = [dense] + walls
    # by paths alone the four are equal: arrival order, one round
    taken, left = S.plan_round(q, sizes, 64, 1 << 24, max_paths=1 << 24, policy="light_first", now=1.1)
    assert taken == q and left == []
    # by layers the wall views go first, and the dense view (150 x 262144
    # > 8 x 262144) stays out of their round
    taken, left = S.plan_round(q, sizes, 64, 1 << 24, max_paths=1 << 24, policy="light_first", now=1.1,
                               layers=layers)
    assert taken == walls and left == [dense]
    taken, left = S.plan_round(left, sizes, 64, 1 << 24, max_paths=1 << 24, policy="light_first", now=1.1,
                               layers=layers)
    assert taken == [dense]
    # unmeasured scenes and cameras weigh 1
    assert S.path_weight(dense, None) == 1.0 and S.path_weight(S.Request("b", 0), layers) == 1.0
    assert S.path_weight(dense, layers) == 150.0


def test_forward_requests_take_slices_of_their_passes():
    sizes = {"a": [(64, 64), (4, 4)]}
    big = S.Request("a", 0, passes=4)                    # 16384 paths
    small = S.Request("a", 1, passes=2)                  # 32 paths
    grad = S.Request("a", 0, kind="gradient", passes=4, target=None)
    taken, left = S.plan_round([big, small], sizes, 64, 10 ** 6, max_paths=4096 + 32, slices=True)
    assert taken == [big, small] and left == []
    assert big.round_passes == 1 and small.round_passes == 0   # one pass of the big one, all of the small
    # a request over the cap that does not come first waits (no slice in another's round)
    taken, left = S.plan_round([small, big], sizes, 64, 10 ** 6, max_paths=4096, slices=True)
    assert taken == [small] and left == [big]
    big.next_pass = 3                                        # one pass left: fits whole
    taken, _ = S.plan_round([big], sizes, 64, 10 ** 6, max_paths=4096, slices=True)
    assert taken == [big] and big.round_passes == 0
    # a gradient request is not sliced by default; as the first of a round it goes whole
    taken, left = S.plan_round([grad, small], sizes, 64, 10 ** 6, max_paths=4096, slices=True)
    assert taken == [grad] and grad.round_passes == 0 and left == [small]
    # with slice_gradients its forward renders in slices like a forward request's
    taken, left = S.plan_round([grad, small], sizes, 64, 10 ** 6, max_paths=4096, slices=True,
                               slice_gradients=True)
    assert taken == [grad] and grad.round_passes == 1
    # without slices the big request waits for a round of its own
    big.next_pass = 0
    taken, left = S.plan_round([small, big], sizes, 64, 10 ** 6, max_paths=4096)
    assert taken == [small] and left == [big]
