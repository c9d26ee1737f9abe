"""The training loop's L2 image loss computed by the post-process
(pale_render_forward_loss / DeviceFrame.forward_loss) against
compute_l2_grad / compute_l2_loss (python/losses.py:10-45) restated in
numpy on the same rendered image."""
import numpy as np
import pytest

from differentiablepointrendering_b200.pale import Renderer
from differentiablepointrendering_b200.scene import make_box_scene

pytestmark = pytest.mark.gpu

SETTINGS = {"photons": 50000, "bounces": 3, "forward_passes": 1, "gather_passes": 2, "adjoint_bounces": 3,
            "adjoint_passes": 1, "gather_radius": 0.02, "rng_mode": "decorrelated"}


def reference_loss(img_rgb, tgt):
    """compute_l2_grad / compute_l2_loss in float32 numpy, as training.py applies them per camera."""
    diff = img_rgb - tgt
    return (diff / diff.size).astype(np.float32), float(0.5 * np.mean(diff * diff))


@pytest.mark.parametrize("channels", [3, 4])
def test_host_forward_loss(gpu, channels):
    sc = make_box_scene(3000, cameras=2, resolution=40)
    r = Renderer.from_scene(sc, SETTINGS)
    try:
        rng = np.random.default_rng(5)
        names = r.get_camera_names()
        targets = {n: rng.uniform(0, 1, (40, 40, channels)).astype(np.float32) for n in names}
        plain = r.render_forward()
        images, dldi, loss = r.render_forward_loss(targets)
        for n in names:
            np.testing.assert_array_equal(images[n], plain[n])          # same seeds, same image
            np.testing.assert_array_equal(images[n + "_raw"], plain[n + "_raw"])
            g, l = reference_loss(images[n][..., :3], targets[n][..., :3])
            np.testing.assert_array_equal(dldi[n], g)
            exact = 0.5 * np.mean((images[n][..., :3].astype(np.float64) - targets[n][..., :3]) ** 2)
            assert loss[n] == pytest.approx(exact, rel=1e-6)
            assert loss[n] == pytest.approx(l, rel=1e-5)
        with pytest.raises(RuntimeError):
            r.render_forward_loss({"no_such_camera": targets[names[0]]})
        with pytest.raises(RuntimeError):
            r.render_forward_loss({names[0]: targets[names[0]][:20]})
    finally:
        r.close()


def test_device_forward_loss_matches_host(gpu):
    import torch

    from differentiablepointrendering_b200.device import DeviceFrame, l2_grad_

    sc = make_box_scene(3000, cameras=3, resolution=32)
    r = Renderer.from_scene(sc, SETTINGS)
    try:
        names = r.get_camera_names()
        rng = np.random.default_rng(9)
        targets = {n: rng.uniform(0, 1, (32, 32, 3)).astype(np.float32) for n in names}
        images, dldi, loss = r.render_forward_loss(targets)
        f = DeviceFrame(r, device=torch.device("cuda:0"))
        packed = torch.from_numpy(np.concatenate([targets[n].reshape(-1, 3) for n in names])).cuda()
        dl = f.forward_loss(packed)
        torch.cuda.synchronize()
        for i, (n, d) in enumerate(zip(names, f.split(f.dldi))):
            np.testing.assert_array_equal(d[..., :3].cpu().numpy(), dldi[n])
            assert float(dl[i]) == loss[n]
            assert float(d[..., 3].abs().max()) == 0.0
        # the torch-op version of the same gradient, camera by camera (torch
        # divides by a scalar through its reciprocal: within one rounding)
        torch_dldi = torch.zeros_like(f.dldi)
        l2_grad_(torch_dldi, f.ldr, packed, f.sizes)
        torch.testing.assert_close(torch_dldi[:, :3], f.dldi[:, :3], rtol=2.4e-7, atol=0)
    finally:
        r.close()


def test_large_host_copies_are_exact(gpu):
    """Host calls whose copies go through the pinned stage (4 MB and more:
    two 512x512 views, 80k surfels' gradients) return byte for byte what
    the device-resident calls leave on the device, and the dL/dI views that
    render_forward_loss returns go back to render_backward in place with the
    same gradients as packed copies of them."""
    import torch

    from differentiablepointrendering_b200.device import DeviceFrame

    sc = make_box_scene(80000, cameras=2, resolution=512)
    r = Renderer.from_scene(sc, SETTINGS)
    try:
        names = r.get_camera_names()
        rng = np.random.default_rng(11)
        targets = {n: rng.uniform(0, 1, (512, 512, 3)).astype(np.float32) for n in names}
        images, dldi, loss = r.render_forward_loss(targets)
        f = DeviceFrame(r, device=torch.device("cuda:0"))
        packed = torch.from_numpy(np.concatenate([targets[n].reshape(-1, 3) for n in names])).cuda()
        dl = f.forward_loss(packed)
        torch.cuda.synchronize()
        for i, (n, l4, d4) in enumerate(zip(names, f.split(f.ldr), f.split(f.dldi))):
            np.testing.assert_array_equal(l4.cpu().numpy(), images[n])
            np.testing.assert_array_equal(d4[..., :3].cpu().numpy(), dldi[n])
            assert float(dl[i]) == loss[n]
            assert dldi[n].strides == (16 * 512, 16, 4)      # an RGB view of the packed buffer
        g_inplace, src = r.render_backward(dldi)
        g_copied, _ = r.render_backward({n: np.ascontiguousarray(v) for n, v in dldi.items()})
        for n in names:
            assert np.all(src["adjoint_source"][n][..., 3] == 1.0)
            np.testing.assert_array_equal(src["adjoint_source"][n][..., :3], dldi[n])
        for k in g_inplace:
            a, b = g_inplace[k].astype(np.float64), g_copied[k].astype(np.float64)
            # the same inputs; the adjoint adds its gradients with float atomics
            assert np.linalg.norm(a - b) <= 1e-5 * max(np.linalg.norm(b), 1e-30), k
        assert np.linalg.norm(g_inplace["opacity"]) > 0
        # the staged gradient copy against the device-resident backward
        f.backward()
        torch.cuda.synchronize()
        dev = f.grads["opacity"].cpu().numpy().astype(np.float64)
        assert np.linalg.norm(dev - g_inplace["opacity"]) <= 1e-5 * np.linalg.norm(dev)
    finally:
        r.close()
