"""Known answers for the oracle's scene queries (the checker of the CUDA
queries in test_gpu_parity.py)."""
import numpy as np

from differentiablepointrendering_b200.scene import empty_points, make_box_scene
from oracle_lib import OracleRenderer

SETTINGS = {"photons": 20000, "bounces": 4, "forward_passes": 1, "gather_passes": 2, "gather_radius": 0.02}


def two_surfels(opacity=(0.5, 0.3)):
    """Two surfels facing +-z at z = 0 and z = 0.1, radius 0.05, beta 0."""
    p = empty_points(2)
    p["position"][:] = [[0, 0, 0], [0, 0, 0.1]]
    p["tangent_u"][:] = [1, 0, 0]
    p["tangent_v"][:] = [0, 1, 0]
    p["scale"][:] = 0.05
    p["albedo"][:] = 0.5
    p["opacity"][:] = opacity
    return make_box_scene(2, cameras=1, resolution=32, points=p)


def test_transmittance_through_two_surfels():
    """intersectBLASPointCloudTransmit: at a surfel's centre alpha_geom =
    (1 - 0)^(4 e^0) = 1, so T = (1 - 0.5)(1 - 0.3).  The closest mesh hit
    is the emitter quad (instance 5, z = 0.499, |x|, |y| <= 0.125) or, off
    its footprint, the ceiling (instance 1, z = 0.5)."""
    sc = two_surfels()
    o = OracleRenderer(sc, SETTINGS)
    try:
        orig = np.array([[0, 0, -0.3], [0.2, 0.2, -0.3], [0, 0, 0.05]], np.float32)
        d = np.array([[0, 0, 1], [0, 0, 1], [0, 0, 1]], np.float32)
        inst, t, T = o.trace_transmittance(orig, d)
        np.testing.assert_allclose(T, [0.5 * 0.7, 1.0, 0.7], rtol=1e-6)
        assert list(inst) == [5, 1, 5]
        np.testing.assert_allclose(t, [0.799, 0.8, 0.449], rtol=1e-5)
        # the walk stops once T <= 0.001: after the first of two surfels of
        # opacity 0.9995 the product is 5e-4, and the second is not applied
        stack = OracleRenderer(two_surfels((0.9995, 0.9995)), SETTINGS)
        _, _, T2 = stack.trace_transmittance(orig[:1], d[:1])
        stack.close()
        np.testing.assert_allclose(T2, [1.0 - np.float32(0.9995)], rtol=1e-4)
    finally:
        o.close()


def test_render_gather_reproduces_forward():
    o = OracleRenderer(make_box_scene(2000, cameras=2, resolution=40), SETTINGS)
    try:
        a = o.render_forward()
        b = o.render_gather()
        for k in a:
            np.testing.assert_array_equal(a[k], b[k])
    finally:
        o.close()
