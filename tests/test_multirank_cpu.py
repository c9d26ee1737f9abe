"""The multi-GPU plumbing (differentiablepointrendering_b200.multigpu) with
two gloo ranks on the CPU.  The cameras of one scene are split over the
ranks (shard_cameras); each rank renders its cameras with the oracle (the
renders are independent given the surfels and the counter-keyed photon map,
which every rank traces identically) and the gradient arrays are summed
with one all-reduce.  The sum must equal one process rendering every camera,
and each rank's images must equal that process's images of its cameras.
The N > 1 GPU path runs the same code over NCCL."""
import math
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from differentiablepointrendering_b200.multigpu import reduce_gradients, shard_cameras, view_offset
from differentiablepointrendering_b200.scene import POINT_FIELDS, make_box_scene, make_surfels, ring_cameras

SETTINGS = {"photons": 5000, "bounces": 3, "forward_passes": 1, "gather_passes": 2, "adjoint_bounces": 3,
            "adjoint_passes": 2, "gather_radius": 0.03, "rng_mode": "decorrelated", "camera_seeds": "camera"}
CAMERAS = 5          # not a multiple of the world size: the shards differ in size


def _scene():
    return make_box_scene(800, cameras=CAMERAS, resolution=24, points=make_surfels(800, 1234))


def render_cameras(names):
    """Images and gradients (asset order) of the given cameras: one oracle
    forward and one adjoint over just these cameras."""
    from oracle_lib import OracleRenderer

    sc = _scene()
    o = OracleRenderer(sc, SETTINGS, threads=1)
    try:
        imgs = o.render_forward(names)
        dl = {n: ((imgs[n + "_raw"][..., :3] - 0.1) / imgs[n + "_raw"][..., :3].size).astype(np.float32)
              for n in names}
        g, _ = o.render_backward(dl)
        order = o.get_point_order()
        out = {}
        for k in POINT_FIELDS:
            a = np.empty_like(g[k])
            a[order] = g[k]
            out[k] = a
        return imgs, out
    finally:
        o.close()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def rank_gradients(rank, world):
    """Rank `rank`'s shard of the scene's cameras: images and gradients."""
    names = shard_cameras([f"camera{k}" for k in range(CAMERAS)], rank, world)
    return render_cameras(names)


def _worker(rank, world, port, outdir, leave_early):
    import datetime
    import sys

    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        imgs, local = rank_gradients(rank, world)
        if leave_early and rank == 1:
            return      # leaves between steps, without joining the collective
        grads = {k: torch.from_numpy(v.copy()) for k, v in local.items()}
        try:
            reduce_gradients(grads)
            status = "ok"
        except Exception as e:  # the peer is gone: the collective must fail, not hang
            status = "error: " + type(e).__name__
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), status=status,
                 **{"local_" + k: v for k, v in local.items()}, **{"sum_" + k: grads[k].numpy() for k in grads},
                 **{"img_" + k: v for k, v in imgs.items()})
    finally:
        if not (leave_early and rank == 1):
            try:
                dist.destroy_process_group()
            except Exception:
                pass


def _run(leave_early):
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_worker, args=(2, _free_port(), d, leave_early), nprocs=2, join=True,
                           start_method="spawn")
        return {r: dict(np.load(os.path.join(d, f"rank{r}.npz"))) for r in range(2)
                if os.path.exists(os.path.join(d, f"rank{r}.npz"))}


def test_view_offsets_interleave_into_one_ring():
    world = 4
    angles = []
    for r in range(world):
        for x, y, _ in ring_cameras(3, offset=view_offset(r, world)):
            angles.append(math.atan2(x, -y) % (2 * math.pi))
    angles = np.sort(angles)
    np.testing.assert_allclose(np.diff(angles), 2 * math.pi / 12, atol=1e-9)
    with pytest.raises(ValueError):
        view_offset(4, 4)


def test_shard_cameras_round_robin():
    names = [f"c{k}" for k in range(5)]
    assert shard_cameras(names, 0, 2) == ["c0", "c2", "c4"]
    assert shard_cameras(names, 1, 2) == ["c1", "c3"]
    assert sorted(sum((shard_cameras(names, r, 3) for r in range(3)), [])) == names
    with pytest.raises(ValueError):
        shard_cameras(names, 2, 2)


def test_sharded_ranks_equal_one_process_over_all_cameras():
    out = _run(leave_early=False)
    assert set(out) == {0, 1}
    for r in (0, 1):
        assert str(out[r]["status"]) == "ok"
    imgs, full = render_cameras([f"camera{k}" for k in range(CAMERAS)])
    # each rank's images are the single process's images of its cameras
    for r in (0, 1):
        for k, v in out[r].items():
            if k.startswith("img_"):
                np.testing.assert_array_equal(v, imgs[k[4:]], err_msg=k)
    for k in POINT_FIELDS:
        a, b = out[0]["sum_" + k].astype(np.float64), full[k].astype(np.float64)
        np.testing.assert_array_equal(out[0]["sum_" + k], out[1]["sum_" + k])
        if k == "opacity":
            assert np.linalg.norm(b) > 0
        # the same terms, summed per rank first: float rounding only
        assert np.linalg.norm(a - b) <= 1e-5 * max(np.linalg.norm(b), 1e-30), k
    # the shards are different cameras: their gradients differ
    assert not np.allclose(out[0]["local_opacity"], out[1]["local_opacity"])


def test_rank_that_leaves_fails_the_collective_with_an_error():
    out = _run(leave_early=True)
    assert 1 not in out
    assert str(out[0]["status"]).startswith("error")
