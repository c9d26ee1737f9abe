"""The C3a gradient check: central finite differences of the L2 image loss
against a gradient, on 64 surfel parameters drawn across the seven groups.

Parameters are taken in each surfel's own frame (U, V its tangents, n the
normal): opacity, beta, albedo r/g/b, scale u/v, and for position,
tangent_u and tangent_v the directions U/|U|, V/|V| (in the surfel's
plane) and n (out of it).  A step in the plane changes the surfels'
alpha_geom where rays hit them; a step out of it also moves the hit points
against the photons deposited there, which a derivative with the photon
map held does not follow, so those three are reported apart.

The finite difference of parameter p is D(eps) = (L(p + eps) - L(p - eps))
/ 2 eps with eps = 1e-3 on the float32 parameters as the renderer holds
them (apply_point_optimization: the tangents as given, the LBVH of the base
render), L the L2 loss of the RAW image of the camera gather against the
target (render_gather: the photon map of the base render held).  The
surfels are about 0.01 across, so a step of 1e-3 is a tenth of one and
D(eps) carries a truncation error of a few percent where alpha_geom curves
(scale, position); Richardson's extrapolation (4 D(eps/2) - D(eps)) / 3
removes its leading term and is the reference the gradient is held to."""
from __future__ import annotations

import numpy as np

GROUPS = ("opacity", "beta", "albedo", "scale", "position", "tangent_u", "tangent_v")
FRAME_GROUPS = ("position", "tangent_u", "tangent_v")
EPS = 1e-3


def _frame(points, i):
    U = points["tangent_u"][i].astype(np.float64)
    V = points["tangent_v"][i].astype(np.float64)
    n = np.cross(U, V)
    return U / np.linalg.norm(U), V / np.linalg.norm(V), n / np.linalg.norm(n)


def draw(points, visible, count=64, seed=99):
    """[(group, surfel, component, direction or None, out_of_plane)]: the
    groups in turn, a surfel among `visible` and a component drawn with
    `seed` (surfel indices in the order of `points`)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        g = GROUPS[k % len(GROUPS)]
        i = int(visible[rng.integers(len(visible))])
        if g in FRAME_GROUPS:
            c = int(rng.integers(3))
            out.append((g, i, c, _frame(points, i)[c], c == 2))
        else:
            width = {"opacity": 1, "beta": 1, "albedo": 3, "scale": 2}[g]
            out.append((g, i, int(rng.integers(width)), None, False))
    return out


def component(grads, p):
    """The gradient's value along parameter p (gradients in the order of
    the points the parameters were drawn from)."""
    g, i, c, d, _ = p
    a = np.asarray(grads[g], np.float64).reshape(len(grads[g]), -1)
    return float(a[i] @ d) if d is not None else float(a[i, c])


def perturbed(points, p, step):
    g, i, c, d, _ = p
    q = {k: v.copy() for k, v in points.items()}
    a = q[g].reshape(len(q[g]), -1)
    if d is not None:
        a[i] = (a[i].astype(np.float64) + step * d).astype(np.float32)
    else:
        a[i, c] = np.float32(a[i, c] + step)
    return q


def l2_loss(img, target):
    d = img.astype(np.float64) - target
    return float(0.5 * np.mean(d * d))


def finite_differences(loss_at, points, params, eps=EPS):
    """(D(eps), Richardson's (4 D(eps/2) - D(eps)) / 3) of loss_at(points)
    along every parameter; loss_at is left at `points`."""
    def central(p, h):
        return (loss_at(perturbed(points, p, h)) - loss_at(perturbed(points, p, -h))) / (2 * h)

    plain, extra = [], []
    for p in params:
        d1, d2 = central(p, eps), central(p, eps / 2)
        plain.append(d1)
        extra.append((4 * d2 - d1) / 3)
    loss_at(points)
    return np.asarray(plain), np.asarray(extra)


def agreement(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))
    rel = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    return cos, rel
