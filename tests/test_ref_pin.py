"""Pins the C oracle to the reference's own kernel code.

oracle/_ref/libpale_ref.so is the reference renderer's unmodified kernel
sources (Pale/Renderer/Kernels/PrimalKernels.cpp, AdjointKernels.cpp,
PostprocessKernel.cpp and their headers) compiled for the CPU against the
project's host SYCL subset, driven by the host flow of SyclBridge.cpp
(submitPhotonMappingKernel, submitAdjointKernel) restated in
oracle/ref_driver.cpp.  Its parallel_for bodies run one after another, so its
atomic queue appends, photon deposits and gradient additions happen in the
order a sequential run of the reference gives, which is the order the
oracle restates.  Both are compiled without contraction of multiply-adds, so
they must agree bit for bit: photon records, grid cells and the cell-sorted
photon order, raw and LDR images, opacity gradients and the number of ray
segments of every stage.

Scenes: the synthetic box (two cameras, so that the per-camera seed stream
is exercised), the reference's own GradientTests scenes `empty` and
`simple_1`, and the box with transmission, absorption and early Russian
roulette switched on so that every branch of the adjoint walk is taken.
The library is built from the reference checkout named by
REFERENCE_CHECKOUT (or used prebuilt); without either these tests skip.
"""
import numpy as np
import pytest

import ref_lib
from fixtures import gradient_test_scene
from oracle_lib import OracleRenderer
from differentiablepointrendering_b200.scene import make_box_scene

pytestmark = pytest.mark.skipif(not ref_lib.available(), reason="reference kernels not built (REFERENCE_CHECKOUT)")

BOX = {"photons": 20000, "bounces": 4, "forward_passes": 1, "gather_passes": 2, "adjoint_bounces": 4,
       "adjoint_passes": 2, "gather_radius": 0.03}


def _box(cams=2, res=40, n=3000):
    return make_box_scene(n, cameras=cams, resolution=res)


def _gradient_scene(case, res=64):
    sc = gradient_test_scene(case, "initial")
    sc.camera_size = np.full_like(sc.camera_size, res)
    return sc


CASES = {
    "box": (_box, BOX),
    "empty": (lambda: _gradient_scene("empty"), {"photons": 50000, "bounces": 5, "forward_passes": 2,
                                                 "gather_passes": 1, "adjoint_bounces": 2, "adjoint_passes": 2,
                                                 "gather_radius": 0.05}),
    "simple_1": (lambda: _gradient_scene("simple_1"), {"photons": 50000, "bounces": 5, "forward_passes": 1,
                                                       "gather_passes": 2, "adjoint_bounces": 3,
                                                       "adjoint_passes": 1, "gather_radius": 0.05}),
    "box_transmit": (lambda: _box(cams=1, res=48), dict(BOX, q_null=0.3, q_reflect=0.4, q_transmit=0.2, rr_start=3,
                                                        seed=7, random_number=99)),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def pair(request):
    make, st = CASES[request.param]
    scene = make()
    ref = ref_lib.ReferenceRenderer(scene, st)
    orc = OracleRenderer(scene, st, threads=1)
    fr, fo = ref.render_forward(), orc.render_forward()
    so = orc.stats()
    yield request.param, scene, ref, orc, fr, fo, so
    ref.close()
    orc.close()


def test_photon_map_bit_exact(pair):
    _, _, ref, orc, _, _, _ = pair
    a, b = ref.get_photons(), orc.get_photons()
    assert len(a["position"]) > 0
    assert len(a["position"]) == len(b["position"])
    for k in ("position", "power", "direction", "cell_id", "sorted"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_forward_images_bit_exact(pair):
    name, scene, _, _, fr, fo, _ = pair
    assert sorted(fr) == sorted(fo)
    for k in fr:
        np.testing.assert_array_equal(fr[k], fo[k], err_msg=f"{name}: {k}")
        assert fr[k].size and np.isfinite(fr[k]).all()
    # LDR is the post-process of the raw image (exposure 1, gamma 2.2, clamp), alpha 1
    for cam in scene.camera_names:
        assert np.all(fr[cam][..., 3] == 1.0)
        assert fr[cam][..., :3].max() <= 1.0


def test_opacity_gradients_bit_exact(pair):
    name, scene, ref, orc, fr, _, _ = pair
    dl = {}
    for cam in scene.camera_names:
        raw = fr[cam + "_raw"][..., :3]
        dl[cam] = ((raw - 0.25) / raw.size).astype(np.float32)
    g_ref = ref.render_backward_opacity(dl)
    g_orc, _ = orc.render_backward(dl)
    np.testing.assert_array_equal(ref.get_point_order(), orc.get_point_order())
    assert np.abs(g_ref).max() > 0, name
    np.testing.assert_array_equal(g_ref, g_orc["opacity"], err_msg=name)


def test_segment_counts_equal(pair):
    _, scene, ref, orc, _, _, so = pair
    photon_segments, _ = ref.segments()
    assert photon_segments == so["photon_segments"]
    assert ref.count_gather_segments() == so["gather_segments"]
    dl = {cam: np.full(tuple(scene.camera_size[i][::-1]) + (3,), 1e-3, np.float32)
          for i, cam in enumerate(scene.camera_names)}
    ref.render_backward_opacity(dl)
    orc.render_backward(dl)
    assert ref.segments()[1] == orc.stats()["adjoint_segments"]
