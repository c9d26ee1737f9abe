"""Batched views: several scenes and views of uneven resolution, passes and
depth in one camera-gather wavefront and one adjoint wavefront
(device.ViewBatch, pale_render_views_*_device).

- Views of one scene with their own passes and adjoint bounces match the
  oracle rendering the same views (images to 1e-4 per pixel as the other
  parity tests, gradients at cosine >= 0.99 and relative L2 <= 1e-2).
- Views of two scenes rendered together equal each scene rendered alone:
  images bit for bit, gradients up to the order of float atomic additions
  (camera-keyed seeds, so a view's samples do not depend on its batch).
"""
import numpy as np
import pytest

from differentiablepointrendering_b200.pale import Renderer
from differentiablepointrendering_b200.scene import make_box_scene, make_surfels
from oracle_lib import OracleRenderer

pytestmark = pytest.mark.gpu

ST = {"photons": 20000, "bounces": 4, "forward_passes": 1, "gather_passes": 4, "adjoint_bounces": 4,
      "adjoint_passes": 4, "gather_radius": 0.03, "rng_mode": "decorrelated", "camera_seeds": "camera"}


def to_asset(values, order):
    out = np.empty_like(values)
    out[order] = values
    return out


def _agree(a, b):
    a = a.astype(np.float64).reshape(-1)
    b = b.astype(np.float64).reshape(-1)
    return float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b))), float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _scene(n, cams, res, seed):
    return make_box_scene(n, cameras=cams, resolution=res, points=make_surfels(n, seed))


def test_views_with_own_passes_and_depth_match_oracle(gpu):
    import torch
    from differentiablepointrendering_b200.device import ViewBatch

    sc = _scene(3000, 3, 48, 1234)
    r = Renderer.from_scene(sc, ST)
    o = OracleRenderer(sc, ST, bvh_kind=0)
    try:
        views = [(0, 2, 1, 0), (0, 0, 3, 2), (0, 1, 4, 1)]
        b = ViewBatch([r], views)
        b.forward_loss(None)
        torch.cuda.synchronize()
        ref = o.render_views([v[1] for v in views], [v[2] for v in views])
        dls = []
        for k, (ldr, raw) in enumerate(ref):
            g_raw = b.split(b.raw)[k].cpu().numpy()
            g_ldr = b.split(b.ldr)[k].cpu().numpy()
            for a, c in ((g_raw[..., :3], raw[..., :3]), (g_ldr[..., :3], ldr[..., :3])):
                rel = np.abs(a - c) / np.maximum(np.abs(c), 1e-3)
                assert np.median(rel) < 1e-4, (k, float(np.median(rel)))
            dls.append(((raw[..., :3] - 0.5 * raw[..., :3].mean()) / raw[..., :3].size).astype(np.float32))
        packed = torch.from_numpy(np.concatenate([np.concatenate([d, np.zeros(d.shape[:2] + (1,), np.float32)], -1)
                                                  .reshape(-1, 4) for d in dls])).cuda()
        g = b.backward(packed)[0]
        torch.cuda.synchronize()
        go = o.backward_views([v[1] for v in views], [v[2] for v in views], [v[3] for v in views], dls)
        cos, rel = _agree(to_asset(g["opacity"].cpu().numpy(), r.get_point_order()),
                          to_asset(go["opacity"], o.get_point_order()))
        assert cos >= 0.99 and rel <= 1e-2, (cos, rel)
    finally:
        r.close()
        o.close()


def test_two_scenes_in_one_wavefront_equal_each_alone(gpu):
    import torch
    from differentiablepointrendering_b200.device import DeviceFrame, ViewBatch

    a_sc, b_sc = _scene(4000, 2, 40, 11), _scene(6000, 3, 56, 22)
    ra, rb = Renderer.from_scene(a_sc, ST), Renderer.from_scene(b_sc, ST)
    try:
        views = [(1, 2, 4, 0), (0, 0, 4, 0), (1, 0, 4, 0), (0, 1, 4, 0)]
        batch = ViewBatch([ra, rb], views)
        batch.forward_loss(None)
        torch.cuda.synchronize()
        alone = {}
        for k, r in enumerate((ra, rb)):
            f = DeviceFrame(r)
            f.forward()
            torch.cuda.synchronize()
            for c, img in enumerate(f.split(f.raw)):
                alone[(k, c)] = (img.cpu().numpy(), f.split(f.ldr)[c].cpu().numpy())
        for i, (s, c, _, _) in enumerate(views):
            np.testing.assert_array_equal(batch.split(batch.raw)[i].cpu().numpy(), alone[(s, c)][0])
            np.testing.assert_array_equal(batch.split(batch.ldr)[i].cpu().numpy(), alone[(s, c)][1])
        # gradients: the batch's per-scene arrays against each scene's own adjoint of its views
        dl = torch.zeros(batch.pixels, 4, device="cuda")
        dl[:, :3] = (batch.raw[:, :3] - 0.3) / batch.pixels
        grads = batch.backward(dl)
        torch.cuda.synchronize()
        for k, r in enumerate((ra, rb)):
            mine = [(i, c) for i, (s, c, _, _) in enumerate(views) if s == k]
            f = DeviceFrame(r, cameras=[c for _, c in mine])
            parts = []
            for i, _ in mine:
                off = sum(w * h for w, h in batch.sizes[:i])
                w, h = batch.sizes[i]
                parts.append(dl[off:off + w * h])
            g1 = f.backward(torch.cat(parts).contiguous())
            torch.cuda.synchronize()
            for key in ("opacity",):
                cos, rel = _agree(grads[k][key].cpu().numpy(), g1[key].cpu().numpy())
                assert cos >= 0.99999 and rel <= 1e-4, (k, key, cos, rel)
    finally:
        ra.close()
        rb.close()


def test_five_scenes_in_one_wavefront_equal_each_alone(gpu):
    """Five scenes in one call stage fewer top nodes each (the call's
    staged-node budget split over its scenes) than a scene alone: the images
    are still those of each scene rendered alone, bit for bit."""
    import torch
    from differentiablepointrendering_b200.device import DeviceFrame, ViewBatch

    scenes = [_scene(2500 + 700 * k, 2, 32 + 8 * k, 40 + k) for k in range(5)]
    rs = [Renderer.from_scene(sc, ST) for sc in scenes]
    try:
        views = [(k, c, 2 + k % 3, 0) for k in (4, 0, 3, 1, 2) for c in (1, 0)]
        batch = ViewBatch(rs, views)
        batch.forward_loss(None)
        torch.cuda.synchronize()
        for i, (s, c, p, _) in enumerate(views):
            alone = ViewBatch([rs[s]], [(0, c, p, 0)])
            alone.forward_loss(None)
            torch.cuda.synchronize()
            np.testing.assert_array_equal(batch.split(batch.raw)[i].cpu().numpy(), alone.split(alone.raw)[0].cpu().numpy())
    finally:
        for r in rs:
            r.close()
