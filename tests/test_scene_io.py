"""Surfel PLY loading: the custom schema with its frame canonicalisation
and albedo clamp, and the Gaussian-splat schema's conversion to surfels
(PLYPointLoader.ixx:71-97, 144-390)."""
import numpy as np

from differentiablepointrendering_b200.scene import load_surfel_ply, make_surfels, write_surfel_ply


def _write_ascii(path, names, rows):
    with open(path, "w") as f:
        f.write("ply\nformat ascii 1.0\n")
        f.write(f"element vertex {len(rows)}\n")
        for n in names:
            f.write(f"property float {n}\n")
        f.write("end_header\n")
        for r in rows:
            f.write(" ".join(repr(float(x)) for x in r) + "\n")


CUSTOM = ["x", "y", "z", "tu_x", "tu_y", "tu_z", "tv_x", "tv_y", "tv_z", "su", "sv", "albedo_r", "albedo_g",
          "albedo_b", "opacity", "beta", "shape"]


def test_custom_schema_round_trip(tmp_path):
    p = make_surfels(50, 3)
    path = str(tmp_path / "c.ply")
    write_surfel_ply(path, p)
    q = load_surfel_ply(path)
    for k in ("position", "scale", "opacity", "beta"):
        np.testing.assert_allclose(q[k], p[k], rtol=1e-6, atol=1e-7)
    n = np.cross(q["tangent_u"], q["tangent_v"])
    assert np.all(n[:, 2] >= 0)
    np.testing.assert_allclose(np.abs(np.sum(q["tangent_u"] * q["tangent_v"], 1)), 0, atol=1e-6)


def test_custom_schema_canonicalises_frames_and_clamps_albedo(tmp_path):
    rows = [
        # non-orthogonal pair: tv loses its tu component
        [0, 0, 0, 2, 0, 0, 1, 1, 0, 0.1, 0.2, 1.5, -0.5, 0.3, 0.7, 0.2, 0],
        # face-down frame (normal -z): tv flips
        [1, 2, 3, 1, 0, 0, 0, -1, 0, 0.1, 0.1, 0.5, 0.5, 0.5, 0.5, 0, 0],
        # parallel pair with tu off the y axis: tv = y made orthogonal
        [0, 0, 0, 1, 0, 0, 3, 0, 0, 0.1, 0.1, 0.5, 0.5, 0.5, 0.5, 0, 0],
        # parallel pair along y: tv from x
        [0, 0, 0, 0, 1, 0, 0, 2, 0, 0.1, 0.1, 0.5, 0.5, 0.5, 0.5, 0, 0],
    ]
    path = str(tmp_path / "c.ply")
    _write_ascii(path, CUSTOM, rows)
    q = load_surfel_ply(path)
    np.testing.assert_allclose(q["tangent_u"][0], [1, 0, 0], atol=1e-7)
    np.testing.assert_allclose(q["tangent_v"][0], [0, 1, 0], atol=1e-7)
    np.testing.assert_allclose(q["albedo"][0], [1.0, 0.0, 0.3], atol=1e-7)
    np.testing.assert_allclose(q["tangent_v"][1], [0, 1, 0], atol=1e-7)
    np.testing.assert_allclose(q["tangent_v"][2], [0, 1, 0], atol=1e-7)
    np.testing.assert_allclose(q["tangent_u"][3], [0, 1, 0], atol=1e-7)
    np.testing.assert_allclose(np.abs(q["tangent_v"][3]), [1, 0, 0], atol=1e-7)
    assert np.all(np.cross(q["tangent_u"], q["tangent_v"])[:, 2] >= 0)


def test_splat_schema_conversion(tmp_path):
    names = ["x", "y", "z", "f_dc_0", "f_dc_1", "f_dc_2", "opacity", "scale_0", "scale_1",
             "rot_0", "rot_1", "rot_2", "rot_3"]
    s = np.sqrt(0.5)
    rows = [
        [0.1, 0.2, 0.3, 0.5, 0.5, 0.5, 0.0, np.log(0.005), np.log(0.01), 1, 0, 0, 0],     # identity
        [0, 0, 0, 0, 0, 0, np.log(1 / 3), 0.0, 0.0, 2 * s, 0, 0, 2 * s],              # 90 deg about z, |q| = 2
        [0, 0, 0, 0, 0, 0, 100.0, -100.0, 0.0, 1, 0, 0, 0],                          # clamped arguments
    ]
    path = str(tmp_path / "s.ply")
    _write_ascii(path, names, rows)
    q = load_surfel_ply(path)
    np.testing.assert_allclose(q["position"][0], [0.1, 0.2, 0.3], rtol=1e-7)
    np.testing.assert_allclose(q["tangent_u"][0], [1, 0, 0], atol=1e-7)
    np.testing.assert_allclose(q["tangent_v"][0], [0, 1, 0], atol=1e-7)
    np.testing.assert_allclose(q["scale"][0], [0.01, 0.02], rtol=1e-6)
    np.testing.assert_allclose(q["opacity"][:2], [0.5, 0.25], rtol=1e-6)
    np.testing.assert_allclose(q["tangent_u"][1], [0, 1, 0], atol=1e-6)
    np.testing.assert_allclose(q["tangent_v"][1], [-1, 0, 0], atol=1e-6)
    np.testing.assert_allclose(q["opacity"][2], 1 / (1 + np.exp(-20.0)), rtol=1e-6)
    np.testing.assert_allclose(q["scale"][2, 0], 2 * np.exp(-20.0), rtol=1e-5)
    np.testing.assert_array_equal(q["albedo"], np.full((3, 3), 0.8, np.float32))
    np.testing.assert_array_equal(q["beta"], 0)
