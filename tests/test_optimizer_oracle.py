"""The optimizer restatement (tests/optim_oracle.py) against the
reference's own optimizer code, through the golden steps recorded by
tests/golden/make_optimizer_golden.py, and the host-side optimizer
description."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import optimizer_cases as OC  # noqa: E402
from optim_oracle import OptimizerOracle, assert_close_to  # noqa: E402

from differentiablepointrendering_b200 import _native as N  # noqa: E402

GOLDEN = os.path.join(HERE, "golden", "optimizer_steps.npz")


@pytest.mark.parametrize("si", range(len(OC.SCENARIOS)), ids=[s[0] for s in OC.SCENARIOS])
def test_restatement_matches_reference_steps(si):
    name, kind, masked, resets = OC.SCENARIOS[si]
    golden = np.load(GOLDEN)
    o = OptimizerOracle(dict(OC.LR, optimizer_type=kind), mask=masked)
    p = OC.initial_parameters()
    for step in range(OC.STEPS):
        p = o.step(p, OC.step_gradients(si, step), resets[step])
        want = {k: golden[f"{name}/{step}/{k}"] for k in OC.FIELDS}
        # float32 rounding only: the torch kernels may fuse multiply-adds
        assert_close_to(p, want, o.condition, ulps=16)
        # next step from the reference's parameters, so that rounding does
        # not compound through the Gram-Schmidt of near-parallel pairs
        p = want
    # the constraints hold exactly where the projection makes them
    assert np.all((p["scale"] >= np.float32(0.01)) & (p["scale"] <= 1))
    assert np.all((p["beta"] >= -3) & (p["beta"] <= 1))
    n = np.cross(p["tangent_u"], p["tangent_v"])
    assert np.all(n[:, 2] >= -1e-6)


def test_golden_cases_reach_every_projection_branch():
    p = OC.initial_parameters()
    _, cond = __import__("optim_oracle").project(p, (0, 0, 1))
    tu, tv = p["tangent_u"], p["tangent_v"]
    u = tu / np.linalg.norm(tu, axis=1, keepdims=True)
    s = tv - np.sum(tv * u, 1, keepdims=True) * u
    degenerate = np.sum(s * s, 1) < 1e-6
    assert degenerate.sum() >= 8
    assert (np.abs(u[degenerate, 1]) >= 0.9).any() and (np.abs(u[degenerate, 1]) < 0.9).any()
    assert (np.cross(tu, tv)[:, 2] < 0).sum() > 10
    assert (p["scale"] < 0.01).any() and (p["scale"] > 1).any()
    assert (p["beta"] < -3).any() and (p["beta"] > 1).any()
    assert (p["opacity"] < 0).any() and (p["albedo"] > 1).any()


def test_optimizer_description():
    o = N.optimizer_from_config({"optimizer_type": "sgd", "learning_rate_position": 0.5})
    assert (o.type, o.flags, o.momentum) == (N.OPT_SGD, 0, 0.8)
    assert list(o.lr) == [0.5, 1.0e-3, 5.0e-3, 2.5e-3, 5.0e-2, 5.0e-2]
    assert o.opacity_reset < 0 and list(o.reference_dir) == [0, 0, 1]
    o = N.optimizer_from_config({"optimizer_type": "nullgrad_adam", "surfel_mask": True}, opacity_reset=0.1)
    assert (o.type, o.flags) == (N.OPT_MASKED_ADAM, N.OPT_SURFEL_MASK)
    assert (o.beta1, o.beta2, o.eps) == (0.9, 0.999, 1e-8)
    assert o.opacity_reset == pytest.approx(0.1)
    with pytest.raises(ValueError):
        N.optimizer_from_config({"optimizer_type": "lbfgs"})
    with pytest.raises(ValueError):
        N.optimizer_from_config({"learning_rate": 1.0})


def test_optimizer_step_rejects_bad_arguments_without_touching_the_gpu():
    import ctypes as C

    lib = N.load_library()
    o = N.optimizer_from_config({})
    assert lib.pale_optimizer_step(None, C.byref(o), None, None) == -1
    assert lib.pale_optimizer_reset(None) == -1
