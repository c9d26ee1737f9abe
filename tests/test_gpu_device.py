"""Device entry points (DeviceFrame) against the host API.

The device calls run on the caller's CUDA stream; with torch's default
stream (whose handle is NULL) they must be ordered with torch's own
default-stream work, so that the dL/dI computed by torch between the
forward and the adjoint pass reads the finished image."""
import numpy as np
import pytest

from differentiablepointrendering_b200.device import DeviceFrame, l2_grad_
from differentiablepointrendering_b200.pale import Renderer
from differentiablepointrendering_b200.scene import make_box_scene

pytestmark = pytest.mark.gpu

SETTINGS = {"photons": 50000, "bounces": 4, "forward_passes": 1, "gather_passes": 2, "adjoint_bounces": 4,
            "adjoint_passes": 2, "gather_radius": 0.02, "rng_mode": "decorrelated"}


@pytest.mark.parametrize("side_stream", [False, True])
def test_device_frame_matches_host_api(gpu, side_stream):
    import torch

    sc = make_box_scene(5000, cameras=2, resolution=96)
    r = Renderer.from_scene(sc, SETTINGS)
    try:
        dev = torch.device("cuda:0")
        frame = DeviceFrame(r, device=dev)
        target = torch.full((frame.pixels, 3), 0.25, device=dev)
        stream = torch.cuda.Stream() if side_stream else torch.cuda.current_stream(dev)
        with torch.cuda.stream(stream):
            frame.forward()
            l2_grad_(frame.dldi, frame.ldr, target, frame.sizes)
            frame.backward()
            ldr = frame.ldr.clone()
            grads = frame.grads["opacity"].clone()
        torch.cuda.synchronize()
        host = r.render_forward()
        dl, off = {}, 0
        for name, (w, h) in zip(r.get_camera_names(), frame.sizes):
            img = host[name]
            np.testing.assert_array_equal(ldr[off:off + w * h].view(h, w, 4).cpu().numpy(), img)
            dl[name] = ((img[..., :3] - 0.25) / (w * h * 3)).astype(np.float32)
            off += w * h
        g, _ = r.render_backward(dl)
        np.testing.assert_allclose(grads.cpu().numpy(), g["opacity"], rtol=1e-4, atol=1e-9)
    finally:
        r.close()
