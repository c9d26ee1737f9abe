"""Generates tests/golden/density_steps.npz with the reference's density control.

Run in a container that has the reference checkout:

    python tests/golden/make_density_golden.py /path/to/DifferentiablePointRendering

It imports python/density_control.py from the checkout and records, for
the cases of density_cases.py, the indices compute_prune_indices_by_opacity
returns (after np.unique, as training.py:770-774 applies them) and the
prune_indices / new children of densify_points_long_axis_split.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import density_cases as DC  # noqa: E402


def main(ref_root: str):
    sys.path.insert(0, os.path.join(ref_root, "python"))
    import density_control as RDC

    out = {}
    p = DC.points(DC.N_PRUNE, 11)
    for name, mo, uq, frac, keep in DC.PRUNE:
        idx = RDC.compute_prune_indices_by_opacity(torch.tensor(p["opacity"]), min_opacity=mo, use_quantile=uq,
                                                   max_fraction_to_prune=frac, min_points_to_keep=keep)
        out[f"prune/{name}"] = np.unique(np.asarray(idx, np.int64))
    q = DC.points(DC.N_SPLIT, 12)
    imp = DC.importance(DC.N_SPLIT, 13)
    for name, use_imp, budget, min_long, thr in DC.SPLIT:
        args = [torch.nn.Parameter(torch.tensor(q[k])) for k in DC.FIELDS]
        res = RDC.densify_points_long_axis_split(*args, importance=torch.tensor(imp) if use_imp else None,
                                                 max_new_points=budget, min_long_axis_scale=min_long,
                                                 grad_threshold=thr)
        if res is None:
            out[f"split/{name}/prune_indices"] = np.zeros(0, np.int64)
            continue
        out[f"split/{name}/prune_indices"] = np.asarray(res["prune_indices"], np.int64)
        for k in DC.FIELDS:
            out[f"split/{name}/new/{k}"] = np.asarray(res["new"][k], np.float32)
    path = os.path.join(HERE, "density_steps.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, len(out), "arrays")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the reference checkout>")
    main(sys.argv[1])
