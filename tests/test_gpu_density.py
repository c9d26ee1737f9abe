"""Density control on the device (pale_prune_by_opacity,
pale_densify_long_axis_split) against the reference's
python/density_control.py through tests/golden/density_steps.npz: the
chosen indices and the edited asset, bit for bit."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import density_cases as DC  # noqa: E402
import density_oracle as DO  # noqa: E402

from differentiablepointrendering_b200.pale import Renderer  # noqa: E402
from differentiablepointrendering_b200.scene import make_box_scene  # noqa: E402

pytestmark = pytest.mark.gpu

GOLDEN = np.load(os.path.join(HERE, "golden", "density_steps.npz"))
SETTINGS = {"photons": 5000, "bounces": 2, "forward_passes": 1, "gather_passes": 1, "adjoint_bounces": 2,
            "adjoint_passes": 1, "gather_radius": 0.03}


def _renderer(p):
    pts = dict(p, shape=np.zeros(p["opacity"].shape[0], np.float32))
    return Renderer.from_scene(make_box_scene(len(p["opacity"]), cameras=1, resolution=16, points=pts), SETTINGS)


@pytest.mark.parametrize("case", DC.PRUNE, ids=[c[0] for c in DC.PRUNE])
def test_prune_by_opacity(gpu, case):
    name, mo, uq, frac, keep = case
    p = DC.points(DC.N_PRUNE, 11)
    r = _renderer(p)
    try:
        removed = r.prune_by_opacity(mo, use_quantile=uq, max_fraction_to_prune=frac, min_points_to_keep=keep)
        want = GOLDEN[f"prune/{name}"]
        np.testing.assert_array_equal(removed, want)
        mask = np.ones(DC.N_PRUNE, bool)
        mask[want] = False
        assert r.num_points == mask.sum()
        for k in DC.FIELDS:
            np.testing.assert_array_equal(r._asset[k], p[k][mask], err_msg=k)
        r.render_forward()      # the rebuilt LBVH renders
    finally:
        r.close()


@pytest.mark.parametrize("case", DC.SPLIT, ids=[c[0] for c in DC.SPLIT])
def test_densify_long_axis_split(gpu, case):
    name, use_imp, budget, min_long, thr = case
    p = DC.points(DC.N_SPLIT, 12)
    imp = DC.importance(DC.N_SPLIT, 13) if use_imp else None
    r = _renderer(p)
    try:
        parents = r.densify_long_axis_split(imp, max_new_points=budget, min_long_axis_scale=min_long,
                                            grad_threshold=thr)
        want = GOLDEN[f"split/{name}/prune_indices"]
        np.testing.assert_array_equal(parents, want)
        children = {k: GOLDEN[f"split/{name}/new/{k}"] for k in DC.FIELDS}
        expect = DO.apply_split(p, want, children)
        assert r.num_points == DC.N_SPLIT + want.size
        for k in DC.FIELDS:
            np.testing.assert_array_equal(r._asset[k], expect[k], err_msg=k)
        np.testing.assert_array_equal(r._asset["shape"][DC.N_SPLIT - want.size:], 0.0)
        r.render_forward()
    finally:
        r.close()


def test_prune_after_optimizer_steps_uses_the_stepped_parameters(gpu):
    """After an optimizer step the asset mirrors the stepped parameters, so
    the opacities pruned are those the step wrote."""
    import torch

    p = DC.points(DC.N_PRUNE, 11)
    r = _renderer(p)
    try:
        cur = r.get_point_parameters()
        g = {k: torch.zeros(v.size, dtype=torch.float32, device="cuda").reshape(v.shape) for k, v in cur.items()
             if k != "shape"}
        g["opacity"] = torch.from_numpy(np.linspace(-1, 1, DC.N_PRUNE).astype(np.float32)).cuda()
        r.optimizer_step({"optimizer_type": "sgd", "learning_rate_opacity": 0.2}, grads=g)
        torch.cuda.synchronize()
        stepped = r.get_point_parameters()["opacity"]
        removed = r.prune_by_opacity(0.1, use_quantile=True)
        np.testing.assert_array_equal(removed, DO.prune_indices(stepped, 0.1, True, 0.3, 1))
    finally:
        r.close()
