"""The density-control restatement against the reference's own
python/density_control.py, through tests/golden/density_steps.npz."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import density_cases as DC  # noqa: E402
import density_oracle as DO  # noqa: E402

GOLDEN = np.load(os.path.join(HERE, "golden", "density_steps.npz"))


@pytest.mark.parametrize("case", DC.PRUNE, ids=[c[0] for c in DC.PRUNE])
def test_prune_matches_reference(case):
    name, mo, uq, frac, keep = case
    p = DC.points(DC.N_PRUNE, 11)
    got = DO.prune_indices(p["opacity"], mo, uq, frac, keep)
    np.testing.assert_array_equal(got, GOLDEN[f"prune/{name}"])


@pytest.mark.parametrize("case", DC.SPLIT, ids=[c[0] for c in DC.SPLIT])
def test_split_matches_reference(case):
    name, use_imp, budget, min_long, thr = case
    p = DC.points(DC.N_SPLIT, 12)
    imp = DC.importance(DC.N_SPLIT, 13) if use_imp else None
    parents, children = DO.split(p, imp, budget, min_long_axis_scale=min_long, grad_threshold=thr)
    np.testing.assert_array_equal(parents, GOLDEN[f"split/{name}/prune_indices"])
    if parents.size:
        for k in DC.FIELDS:
            np.testing.assert_array_equal(children[k], GOLDEN[f"split/{name}/new/{k}"], err_msg=k)


def test_cases_cover_the_branches():
    assert GOLDEN["prune/abs_none"].size == 0                       # nothing below the threshold
    assert GOLDEN["prune/q50_capped"].size == int(0.3 * DC.N_PRUNE)  # the cap binds
    assert GOLDEN["split/long_budget/prune_indices"].size == 10      # budget by long axis
    assert GOLDEN["split/score_budget/prune_indices"].size == 8      # budget by importance
