"""Generates tests/golden/optimizer_steps.npz with the reference's optimizer code.

Run in a container that has the reference checkout:

    python tests/golden/make_optimizer_golden.py /path/to/DifferentiablePointRendering

It imports python/optimizers.py (create_optimizer, create_masked_optimizer,
MaskedAdam, compute_surfel_update_mask,
assign_numpy_gradients_to_tensors_masked) and python/render_hooks.py
(orthonormalize_tangents_inplace and the verify_* clamps) from the
checkout, with a stand-in for the compiled `pale` module that
render_hooks.py imports but these functions do not use.  For every
scenario of optimizer_cases.py it then takes the steps of the training
loop (python/training.py:685-727): zero_grad, gradients into .grad (masked
where the scenario says so), optimizer.step(), the opacity reset, and
verify_parameters_inplane (training.py:326-343), on CPU float32 tensors,
recording the parameters after every step.
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import optimizer_cases as OC  # noqa: E402


class _Cfg:
    def __init__(self, kind):
        self.optimizer_type = kind
        for k, v in OC.LR.items():
            setattr(self, k, v)


def main(ref_root: str):
    sys.path.insert(0, os.path.join(ref_root, "python"))
    stub = types.ModuleType("pale")
    stub.Renderer = object
    sys.modules.setdefault("pale", stub)
    import optimizers as ROPT
    import render_hooks as RH

    torch.manual_seed(0)
    init = OC.initial_parameters()
    out = {}
    for si, (name, kind, masked, resets) in enumerate(OC.SCENARIOS):
        P = {k: torch.nn.Parameter(torch.tensor(init[k])) for k in OC.FIELDS}
        args = [P[k] for k in OC.FIELDS]
        if kind == "masked_adam":
            opt = ROPT.create_masked_optimizer(_Cfg(kind), *args)
        else:
            opt = ROPT.create_optimizer(_Cfg(kind), *args)
        for step in range(OC.STEPS):
            g = OC.step_gradients(si, step)
            opt.zero_grad(set_to_none=True)
            if masked:
                mask = ROPT.compute_surfel_update_mask(*[g[k] for k in OC.FIELDS])
                ROPT.assign_numpy_gradients_to_tensors_masked(torch.device("cpu"), *args,
                                                              *[g[k] for k in OC.FIELDS], mask)
            else:
                for k in OC.FIELDS:
                    P[k].grad = torch.tensor(g[k], dtype=torch.float32)
            opt.step()
            if resets[step] is not None:
                with torch.no_grad():
                    P["opacity"][:] = resets[step]
            with torch.no_grad():
                RH.orthonormalize_tangents_inplace(P["tangent_u"], P["tangent_v"])
                RH.verify_scales_inplace(P["scale"])
                RH.verify_albedos_inplace(P["albedo"])
                RH.verify_opacities_inplace(P["opacity"])
                RH.verify_beta_inplace(P["beta"])
            for k in OC.FIELDS:
                out[f"{name}/{step}/{k}"] = P[k].detach().numpy().copy()
    path = os.path.join(HERE, "optimizer_steps.npz")
    np.savez_compressed(path, torch_version=np.array(torch.__version__), **out)
    print("wrote", path, len(out), "arrays")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the reference checkout>")
    main(sys.argv[1])
