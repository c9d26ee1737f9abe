"""The reference's finite-difference gradient check, restated.

python/finite_difference/fd_test.py sweeps the opacity of surfel 0 over
i/10, i = 0..10, and compares the adjoint opacity gradient of the L2 loss
on the RAW image (losses.compute_l2_grad: (I - T) / I.size) with a finite
difference of the loss L = mean((I - T)^2) / 2 (central with eps = 5e-3
where [v - eps, v + eps] stays inside [0, 1], one-sided at the ends).  It
sets the value with set_point_opacity(opacity, index) and calls
rebuild_bvh() before every render.  batch_fd_check.py scores every row but
the last: a row passes when |an - fd| <= 1e-4 or |an - fd| / (|an| + |fd|)
<= 0.05, and a case passes when every scored row passes.  The cases are the
`empty` and `simple_1` GradientTests scenes (tests.json); the target image
is a render of the scene's target.ply with the same settings
(render_target.py).
"""
from __future__ import annotations

import numpy as np

from fixtures import gradient_test_points, gradient_test_scene

CAMERA = "camera1"
EPS = 5e-3
ITERATIONS = 10
ABS_THRESHOLD = 1e-4
REL_THRESHOLD = 0.05


def scene(case: str, which: str, res: int | None = None):
    sc = gradient_test_scene(case, "initial")
    if res is not None:
        sc.camera_size = np.full_like(sc.camera_size, res)
    if which != "initial":
        sc = sc.with_points(gradient_test_points(case, which))
    return sc


def raw_rgb(r) -> np.ndarray:
    return np.asarray(r.render_forward()[CAMERA + "_raw"], np.float32)[..., :3]


def l2_loss(img, target) -> float:
    d = img - target
    return float(0.5 * np.mean(d * d))


def sweep(r, target, set_opacity):
    """Returns [(value, analytic, fd)] of fd_test.py's opacity sweep on
    renderer `r`; `set_opacity(r, v)` sets surfel 0 and rebuilds."""
    rows = []
    for it in range(ITERATIONS + 1):
        v = it / ITERATIONS
        set_opacity(r, v)
        l0 = l2_loss(raw_rgb(r), target)
        if v - EPS >= 0.0 and v + EPS <= 1.0:
            set_opacity(r, v + EPS)
            lp = l2_loss(raw_rgb(r), target)
            set_opacity(r, v - EPS)
            lm = l2_loss(raw_rgb(r), target)
            fd = (lp - lm) / (2 * EPS)
        elif v + EPS <= 1.0:
            set_opacity(r, v + EPS)
            fd = (l2_loss(raw_rgb(r), target) - l0) / EPS
        else:
            set_opacity(r, v - EPS)
            fd = (l0 - l2_loss(raw_rgb(r), target)) / EPS
        set_opacity(r, v)
        img = raw_rgb(r)
        grads, _ = r.render_backward({CAMERA: ((img - target) / img.size).astype(np.float32)})
        rows.append((v, float(np.asarray(grads["opacity"]).reshape(-1)[0]), float(fd)))
    return rows


def failing_rows(rows):
    """batch_fd_check.py's scoring: the last row is not scored."""
    bad = []
    for v, an, fd in rows[:-1]:
        abs_err = abs(an - fd)
        rel_err = abs_err / max(1e-12, abs(an) + abs(fd))
        if not (abs_err <= ABS_THRESHOLD or rel_err <= REL_THRESHOLD):
            bad.append((v, an, fd, abs_err, rel_err))
    return bad
