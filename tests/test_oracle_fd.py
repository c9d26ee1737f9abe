"""The reference's own gradient check (fd_harness) run on the oracle.

The reference runs 50 forward passes of 1e6 photons on 500x500.  This run
keeps its bounce counts, adjoint passes and seed and uses 4 passes of 1e6
photons on 200x200 pixels, so that the sweep finishes in about a minute on
the CPU, on the `empty` scene.  With fewer photons the photon-map noise of
the forward image moves the finite difference by more than 5%.  The full
harness with the reference's own settings, `simple_1` included, runs on the
CUDA renderer in test_gpu_fd.py.
"""
import numpy as np

import fd_harness as H
from oracle_lib import OracleRenderer

SETTINGS = {"photons": 1000000, "bounces": 5, "forward_passes": 4, "gather_passes": 1, "adjoint_bounces": 1,
            "adjoint_passes": 8, "seed": 42}
RES = 200


def _set_opacity(r, value):
    p = r.get_point_parameters()
    p["opacity"][0] = value
    r.apply_point_optimization(p)


def test_oracle_opacity_gradient_matches_finite_difference_empty():
    t = OracleRenderer(H.scene("empty", "target", RES), SETTINGS)
    target = H.raw_rgb(t)
    t.close()
    r = OracleRenderer(H.scene("empty", "initial", RES), SETTINGS)
    try:
        rows = H.sweep(r, target, _set_opacity)
    finally:
        r.close()
    assert not H.failing_rows(rows), (H.failing_rows(rows), rows)
    assert max(abs(fd) for _, _, fd in rows) > 1e-3


def test_oracle_null_weight_with_photon_map_held():
    """`simple_1` has a lit wall 0.2 behind its surfel, so the
    NullTransmittance (occlusion) term matters.  With the photon map held
    (render_gather) the finite difference is what the adjoint estimates; it
    agrees within the reference's 5% with null_weight "unbiased", while the
    reference's weighting (the term times qNull = 0.5) overshoots by about
    20%."""
    st = dict(SETTINGS, adjoint_bounces=2, adjoint_passes=32, rng_mode="decorrelated", forward_passes=8)
    res = 150
    t = OracleRenderer(H.scene("simple_1", "target", res), st)
    target = H.raw_rgb(t)
    t.close()
    ratios = {}
    for mode in ("unbiased", "reference"):
        r = OracleRenderer(H.scene("simple_1", "initial", res), dict(st, null_weight=mode))
        try:
            rows = []
            for v in (0.2, 0.5, 0.8):
                _set_opacity(r, v)
                base = H.raw_rgb(r)
                _set_opacity(r, v + H.EPS)
                lp = H.l2_loss(np.asarray(r.render_gather()[H.CAMERA + "_raw"])[..., :3], target)
                _set_opacity(r, v - H.EPS)
                lm = H.l2_loss(np.asarray(r.render_gather()[H.CAMERA + "_raw"])[..., :3], target)
                _set_opacity(r, v)
                g, _ = r.render_backward({H.CAMERA: ((base - target) / base.size).astype(np.float32)})
                rows.append((v, float(g["opacity"][0]), (lp - lm) / (2 * H.EPS)))
            ratios[mode] = [an / fd for _, an, fd in rows]
            if mode == "unbiased":
                assert not H.failing_rows(rows + [rows[-1]]), rows
        finally:
            r.close()
    assert min(ratios["reference"]) > 1.1, ratios
