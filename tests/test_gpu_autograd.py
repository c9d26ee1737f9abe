"""The renderer as a torch.autograd.Function (autograd.render): the
backward pass is the adjoint with the incoming image gradient as dL/dI,
and torch optimizers train through it."""
import numpy as np
import pytest

from differentiablepointrendering_b200.pale import Renderer
from differentiablepointrendering_b200.scene import make_box_scene, make_surfels

pytestmark = pytest.mark.gpu

SETTINGS = {"photons": 100000, "bounces": 3, "forward_passes": 1, "gather_passes": 2, "adjoint_bounces": 3,
            "adjoint_passes": 2, "gather_radius": 0.03, "gradients": "all"}


@pytest.mark.parametrize("output,estimator", [("raw", "reference"), ("ldr", "reference"), ("raw", "gather")])
def test_backward_is_the_adjoint(gpu, output, estimator):
    import torch

    from differentiablepointrendering_b200 import autograd as A
    from differentiablepointrendering_b200.device import DeviceFrame

    r = Renderer.from_scene(make_box_scene(3000, cameras=2, resolution=32), dict(SETTINGS, estimator=estimator))
    try:
        f = DeviceFrame(r, device=torch.device("cuda:0"))
        params = A.parameters(r)
        w = torch.rand(f.pixels, 4, device="cuda", generator=torch.Generator("cuda").manual_seed(3))
        img = A.render(f, params, output=output)
        direct = (f.ldr if output == "ldr" else f.raw).clone()
        torch.testing.assert_close(img, direct, rtol=0, atol=0)
        (img * w).sum().backward()
        auto = {k: v.grad.clone() for k, v in params.items()}
        # the same forward and adjoint through the device entry points
        f.forward()
        g = f.backward(w.contiguous())
        torch.cuda.synchronize()
        for k in A.FIELDS:
            # the same events, added by float atomics in a different order
            want = g[k].reshape(auto[k].shape)
            scale = float(want.abs().max())
            torch.testing.assert_close(auto[k], want, rtol=1e-4, atol=1e-6 * scale, msg=k)
        assert float(auto["opacity"].abs().sum()) > 0 and float(auto["position"].abs().sum()) > 0
    finally:
        r.close()


def test_torch_adam_trains_through_the_renderer(gpu):
    import torch

    from differentiablepointrendering_b200 import autograd as A
    from differentiablepointrendering_b200.device import DeviceFrame

    pts = make_surfels(4000, 77)
    tp = {k: v.copy() for k, v in pts.items()}
    tp["opacity"][:] = 0.9
    st = {k: v.copy() for k, v in pts.items()}
    st["opacity"][:] = 0.2
    settings = dict(SETTINGS, photons=200000, gather_passes=4, adjoint_passes=4, gradients="opacity",
                    rng_mode="decorrelated")
    dev = torch.device("cuda:0")
    t = Renderer.from_scene(make_box_scene(4000, cameras=2, resolution=64, points=tp), settings)
    try:
        tf = DeviceFrame(t, device=dev)
        tf.forward()
        target = tf.raw[:, :3].clone()
    finally:
        t.close()
    r = Renderer.from_scene(make_box_scene(4000, cameras=2, resolution=64, points=st), settings)
    try:
        f = DeviceFrame(r, device=dev)
        params = A.parameters(r)
        for k in A.FIELDS:
            params[k].requires_grad_(k == "opacity")
        opt = torch.optim.Adam([params["opacity"]], lr=0.05)
        losses = []
        for _ in range(12):
            opt.zero_grad()
            img = A.render(f, params)
            loss = 0.5 * ((img[:, :3] - target) ** 2).mean()
            loss.backward()
            opt.step()
            with torch.no_grad():
                params["opacity"].clamp_(0.0, 1.0)
            losses.append(float(loss.detach()))
        assert float(params["opacity"].detach().mean()) > 0.23
        assert np.mean(losses[-3:]) < 0.85 * np.mean(losses[:3]), losses
    finally:
        r.close()
