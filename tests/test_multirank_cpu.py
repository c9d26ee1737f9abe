"""The multi-GPU plumbing (differentiablepointrendering_b200.multigpu) with
two gloo ranks on the CPU.  Each rank renders its own views of the same
surfels with the oracle (the renders are independent given the surfels and
the counter-keyed photon map) and the gradient arrays are summed with one
all-reduce.  The N > 1 GPU path runs the same code over NCCL."""
import math
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from differentiablepointrendering_b200.multigpu import reduce_gradients, view_offset
from differentiablepointrendering_b200.scene import POINT_FIELDS, make_box_scene, make_surfels, ring_cameras

SETTINGS = {"photons": 5000, "bounces": 3, "forward_passes": 1, "gather_passes": 1, "adjoint_bounces": 3,
            "adjoint_passes": 1, "gather_radius": 0.03, "rng_mode": "decorrelated"}
VIEWS_PER_RANK = 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def rank_gradients(rank, world):
    """Opacity-gradient arrays of rank `rank`'s views (asset order)."""
    from oracle_lib import OracleRenderer

    pts = make_surfels(800, 1234)
    sc = make_box_scene(800, cameras=VIEWS_PER_RANK, resolution=24, points=pts,
                        ring_offset=view_offset(rank, world))
    o = OracleRenderer(sc, SETTINGS, threads=1)
    try:
        img = o.render_forward()
        dl = {n: ((img[n + "_raw"][..., :3] - 0.1) / img[n + "_raw"][..., :3].size).astype(np.float32)
              for n in sc.camera_names}
        g, _ = o.render_backward(dl)
        order = o.get_point_order()
        out = {}
        for k in POINT_FIELDS:
            a = np.empty_like(g[k])
            a[order] = g[k]
            out[k] = a
        return out
    finally:
        o.close()


def _worker(rank, world, port, outdir, leave_early):
    import datetime
    import sys

    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        local = rank_gradients(rank, world)
        if leave_early and rank == 1:
            return      # leaves between steps, without joining the collective
        grads = {k: torch.from_numpy(v.copy()) for k, v in local.items()}
        try:
            reduce_gradients(grads)
            status = "ok"
        except Exception as e:  # the peer is gone: the collective must fail, not hang
            status = "error: " + type(e).__name__
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), status=status,
                 **{"local_" + k: v for k, v in local.items()}, **{"sum_" + k: grads[k].numpy() for k in grads})
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


def test_gradients_summed_over_two_ranks():
    out = _run(leave_early=False)
    assert set(out) == {0, 1}
    for r in (0, 1):
        assert str(out[r]["status"]) == "ok"
    for k in POINT_FIELDS:
        want = out[0]["local_" + k] + out[1]["local_" + k]
        np.testing.assert_allclose(out[0]["sum_" + k], want, rtol=1e-6, atol=1e-12)
        np.testing.assert_array_equal(out[0]["sum_" + k], out[1]["sum_" + k])
    # the two shards are different views: their gradients differ
    assert not np.allclose(out[0]["local_opacity"], out[1]["local_opacity"])


def test_rank_that_leaves_fails_the_collective_with_an_error():
    out = _run(leave_early=True)
    assert 1 not in out
    assert str(out[0]["status"]).startswith("error")
