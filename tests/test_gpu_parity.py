"""CUDA renderer vs the CPU oracle on identical inputs.

Integer work must match bit-exactly (Morton codes, sort order, LBVH nodes,
photon cell ids and order); floating-point results within the stated
tolerances.  Both sides use the same counter-keyed RNG streams, so whole
renders agree up to ULP-level differences of CUDA's and glibc's sin/cos/
exp/pow, which can make a small fraction of paths diverge.
"""
import numpy as np
import pytest

from differentiablepointrendering_b200.pale import Renderer
from differentiablepointrendering_b200.scene import make_box_scene
from oracle_lib import OracleRenderer, collected_asset_points, lbvh_reference, surfel_aabbs

pytestmark = pytest.mark.gpu

SETTINGS = {"photons": 20000, "bounces": 4, "forward_passes": 1, "gather_passes": 2, "adjoint_bounces": 4,
            "adjoint_passes": 2, "gather_radius": 0.02}


@pytest.fixture(scope="module")
def box():
    return make_box_scene(3000, cameras=2, resolution=64)


@pytest.fixture(scope="module")
def pair(box):
    from conftest import has_gpu
    if not has_gpu():
        pytest.skip("no CUDA device")
    g = Renderer.from_scene(box, SETTINGS)
    o = OracleRenderer(box, SETTINGS, bvh_kind=0)
    yield g, o
    g.close()
    o.close()


def to_asset(values, order):
    out = np.empty_like(values)
    out[order] = values
    return out


@pytest.mark.parametrize("leaf", [1, 4])
def test_lbvh_bit_exact(gpu, box, leaf):
    g = Renderer.from_scene(box, dict(SETTINGS, leaf_size=leaf))
    col = collected_asset_points(box)
    lo, hi = surfel_aabbs(col["position"], col["tangent_u"], col["tangent_v"], col["scale"])
    codes, nodes = g.get_bvh()
    top = nodes.shape[0] - (g.num_points - 1)    # node count = staged top copies + Karras nodes
    codes_ref, order_ref, nodes_ref = lbvh_reference(col["position"], lo, hi, leaf_size=leaf, top=top)
    order = g.get_point_order()
    g.close()
    assert np.array_equal(codes, codes_ref)
    assert np.all(np.diff(codes.astype(np.int64)) >= 0)
    assert np.array_equal(order, order_ref)
    assert nodes.shape == nodes_ref.shape
    assert np.array_equal(nodes.view(np.uint32), nodes_ref.view(np.uint32))


def test_parameters_in_bvh_order(pair, box):
    g, o = pair
    pg = g.get_point_parameters()
    og = g.get_point_order()
    po = o.get_point_parameters()
    oo = o.get_point_order()
    for k in pg:
        np.testing.assert_array_equal(to_asset(pg[k], og), to_asset(po[k], oo), err_msg=k)


def test_closest_hits_match(pair, box):
    g, o = pair
    rng = np.random.default_rng(7)
    n = 20000
    orig = rng.uniform(-0.45, 0.45, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    gi, gp, gt, ga, gx = g.trace_rays(orig, d)
    oi, op, ot, oa, ox = o.trace_rays(orig, d)
    assert np.mean(gi == oi) > 0.999
    same = (gi == oi)
    surf = same & (gi == box.instance_mesh.shape[0])
    # surfel ids compared in asset order
    gid = g.get_point_order()[gp[surf]]
    oid = o.get_point_order()[op[surf]]
    assert np.mean(gid == oid) > 0.999
    hit = same & (gi >= 0)
    np.testing.assert_allclose(gt[hit], ot[hit], rtol=1e-5, atol=1e-6)
    both = surf.copy()
    both[surf] = gid == oid
    np.testing.assert_allclose(ga[both], oa[both], rtol=1e-4, atol=1e-6)
    # integer-exact on the hit-or-miss decision and the instance
    assert np.array_equal(gi >= 0, oi >= 0) or np.mean((gi >= 0) == (oi >= 0)) > 0.9995


def test_transmittance_matches_oracle(pair, box):
    """Transmit-mode queries (intersectBLASPointCloudTransmit): rays from
    inside and outside the box through the cloud."""
    g, o = pair
    rng = np.random.default_rng(8)
    n = 20000
    orig = rng.uniform(-0.45, 0.45, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    gi, gt, gT = g.trace_transmittance(orig, d)
    oi, ot, oT = o.trace_transmittance(orig, d)
    assert np.array_equal(gi, oi)
    hit = gi >= 0
    np.testing.assert_allclose(gt[hit], ot[hit], rtol=1e-5, atol=1e-6)
    # products of (1 - opacity * alpha_geom); CUDA's and glibc's powf/expf
    # differ by ulps, which can flip a grazing surfel in or out of a walk
    close = np.abs(gT - oT) <= 1e-4 + 1e-4 * np.abs(oT)
    assert np.mean(close) > 0.999, np.mean(close)
    assert np.mean(oT < 0.999) > 0.1      # the rays do cross surfels
    assert np.all((gT >= 0.0) & (gT <= 1.0))


def _lookups_close(Eg, Eo):
    """Same photons accepted, summed in another order: within float rounding
    of the sum (1e-5 relative) on all but the rare query where a photon lies
    within a rounding error of the radius or of the cosine cut."""
    scale = np.maximum(np.abs(Eo).max(axis=1, keepdims=True), 1e-30)
    rel = np.abs(Eg - Eo) / scale
    assert np.mean(np.all(rel <= 1e-5, axis=1)) >= 0.999, np.mean(np.all(rel <= 1e-5, axis=1))
    assert np.all(np.isfinite(Eg))
    assert float(np.abs(Eg - Eo).sum()) <= 1e-4 * float(np.abs(Eo).sum())


def test_photon_grid_and_lookup_exact(pair):
    g, o = pair
    rng = np.random.default_rng(3)
    n = 200000
    pos = rng.uniform(-0.5, 0.5, (n, 3)).astype(np.float32)
    pw = rng.uniform(0, 1e-4, (n, 3)).astype(np.float32)
    dr = rng.normal(size=(n, 3))
    dr = (dr / np.linalg.norm(dr, axis=1, keepdims=True)).astype(np.float32)
    g.load_photons(pos, pw, dr)
    o.load_photons(pos, pw, dr)
    pg, po = g.get_photons(), o.get_photons()
    np.testing.assert_array_equal(pg["grid"], po["grid"])
    np.testing.assert_array_equal(pg["cell_id"], po["cell_id"])
    np.testing.assert_array_equal(pg["sorted"], po["sorted"])
    q = rng.uniform(-0.45, 0.45, (5000, 3)).astype(np.float32)
    nq = rng.normal(size=(5000, 3))
    nq = (nq / np.linalg.norm(nq, axis=1, keepdims=True)).astype(np.float32)
    Eg, Eo = g.gather_irradiance(q, nq), o.gather_irradiance(q, nq)
    _lookups_close(Eg, Eo)


def test_dense_lookup_exact(pair):
    """Thousands of photons per query (a dense cluster, as inside a surfel
    cloud): many 32-photon rounds per lookup, still bit-exact."""
    g, o = pair
    rng = np.random.default_rng(4)
    n = 100000
    pos = (rng.normal(size=(n, 3)) * 0.03).astype(np.float32)
    pw = rng.uniform(0, 1e-4, (n, 3)).astype(np.float32)
    dr = rng.normal(size=(n, 3))
    dr = (dr / np.linalg.norm(dr, axis=1, keepdims=True)).astype(np.float32)
    g.load_photons(pos, pw, dr)
    o.load_photons(pos, pw, dr)
    q = (rng.normal(size=(1000, 3)) * 0.03).astype(np.float32)
    nq = rng.normal(size=(1000, 3))
    nq = (nq / np.linalg.norm(nq, axis=1, keepdims=True)).astype(np.float32)
    Eg, Eo = g.gather_irradiance(q, nq), o.gather_irradiance(q, nq)
    assert o.stats()["photons_scanned"] > 1000 * 1000
    _lookups_close(Eg, Eo)


def test_forward_images_match_oracle(pair, box):
    g, o = pair
    ig, io = g.render_forward(), o.render_forward()
    for name in box.camera_names:
        a, b = ig[name + "_raw"][..., :3], io[name + "_raw"][..., :3]
        err = np.abs(a - b)
        scale = np.maximum(np.abs(b), 1e-3)
        assert np.median(err / scale) < 1e-4, name
        assert np.mean(err / scale < 1e-3) > 0.95, name
        assert np.abs(a.mean() - b.mean()) / b.mean() < 1e-2, name
        np.testing.assert_allclose(ig[name][..., 3], 1.0)
    sg, so = g.stats(), o.stats()
    assert abs(sg["photons_stored"] - so["photons_stored"]) <= 0.01 * so["photons_stored"]


def test_forward_is_deterministic(pair, box):
    g, _ = pair
    a = g.render_forward()
    b = g.render_forward()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])


def test_opacity_gradients_match_oracle(pair, box):
    g, o = pair
    ig = g.render_forward()
    o.render_forward()
    tgt = {}
    for name in box.camera_names:
        raw = ig[name + "_raw"][..., :3]
        tgt[name] = ((raw - 0.5 * raw.mean()) / raw.size).astype(np.float32)
    gg, _ = g.render_backward(tgt)
    go, _ = o.render_backward(tgt)
    a = to_asset(gg["opacity"], g.get_point_order()).astype(np.float64)
    b = to_asset(go["opacity"], o.get_point_order()).astype(np.float64)
    cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    assert cos >= 0.99 and rel <= 1e-2, (cos, rel)
    for k in ("position", "tangent_u", "tangent_v", "scale", "albedo", "beta", "shape"):
        assert gg[k].shape[0] == g.num_points


def test_traversal_cost_close_to_oracle(pair, box):
    """Node visits per ray on the GPU stay within 2x of the oracle's on the
    same rays (catches culling regressions that keep results correct)."""
    g, o = pair
    rng = np.random.default_rng(11)
    n = 4000
    orig = rng.uniform(-0.39, 0.39, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    g.trace_rays(orig, d)
    o.trace_rays(orig, d)
    ng, no = g.stats()["node_visits"] / n, o.stats()["node_visits"] / n
    tg, to = g.stats()["surfel_tests"] / n, o.stats()["surfel_tests"] / n
    assert ng <= 2.0 * no + 8, (ng, no)
    assert tg <= 2.0 * to + 8, (tg, to)


def _opacity_agreement(g, o, scene):
    ig = g.render_forward()
    o.render_forward()
    tgt = {}
    for name in scene.camera_names:
        raw = ig[name + "_raw"][..., :3]
        tgt[name] = ((raw - 0.5 * raw.mean()) / raw.size).astype(np.float32)
    gg, _ = g.render_backward(tgt)
    go, _ = o.render_backward(tgt)
    a = to_asset(gg["opacity"], g.get_point_order()).astype(np.float64)
    b = to_asset(go["opacity"], o.get_point_order()).astype(np.float64)
    cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    return cos, rel


def test_decorrelated_passes_match_oracle(gpu, box):
    """Decorrelated seeds: every (camera, pass) job of the batched adjoint
    draws its own streams, keyed by its rank inside its own job."""
    st = dict(SETTINGS, rng_mode="decorrelated", gather_passes=3, adjoint_passes=3)
    g = Renderer.from_scene(box, st)
    o = OracleRenderer(box, st, bvh_kind=0)
    try:
        cos, rel = _opacity_agreement(g, o, box)
        assert cos >= 0.99 and rel <= 1e-2, (cos, rel)
    finally:
        g.close()
        o.close()


def test_adjoint_split_into_batches_matches_oracle(gpu):
    """More jobs than one adjoint batch holds (1024): the second batch must
    pick up the seed table and queues where the first left off."""
    sc = make_box_scene(1500, cameras=1, resolution=8)
    st = dict(SETTINGS, rng_mode="decorrelated", gather_passes=1, adjoint_passes=1100)
    g = Renderer.from_scene(sc, st)
    o = OracleRenderer(sc, st, bvh_kind=0)
    try:
        cos, rel = _opacity_agreement(g, o, sc)
        assert cos >= 0.99 and rel <= 1e-2, (cos, rel)
    finally:
        g.close()
        o.close()


def test_all_gradient_groups_match_oracle(gpu, box):
    """gradients = "all": the six groups beyond opacity (a23 formulas) on the
    GPU equal the oracle's on the same paths."""
    st = dict(SETTINGS, gradients="all", rng_mode="decorrelated", null_weight="unbiased")
    g = Renderer.from_scene(box, st)
    o = OracleRenderer(box, st, bvh_kind=0)
    try:
        ig = g.render_forward()
        o.render_forward()
        tgt = {n: ((ig[n + "_raw"][..., :3] - 0.5 * ig[n + "_raw"][..., :3].mean()) / ig[n + "_raw"][..., :3].size)
               .astype(np.float32) for n in box.camera_names}
        gg, _ = g.render_backward(tgt)
        go, _ = o.render_backward(tgt)
        og, oo = g.get_point_order(), o.get_point_order()
        for k in ("opacity", "beta", "albedo", "scale", "position", "tangent_u", "tangent_v"):
            a = to_asset(gg[k], og).astype(np.float64).reshape(-1)
            b = to_asset(go[k], oo).astype(np.float64).reshape(-1)
            assert np.linalg.norm(b) > 0, k
            cos = a @ b / (np.linalg.norm(a) * np.linalg.norm(b))
            rel = np.linalg.norm(a - b) / np.linalg.norm(b)
            assert cos >= 0.99 and rel <= 1e-2, (k, cos, rel)
    finally:
        g.close()
        o.close()


def test_camera_seeds_by_camera_shard_like_one_call(gpu, box):
    """camera_seeds = "camera" keys a camera's gather and adjoint seeds by
    its scene index: one camera rendered alone equals the oracle's render of
    it, and the gradients of the cameras rendered one call each sum to the
    gradient of one call over all of them (what ranks that split the
    cameras of a scene rely on)."""
    st = dict(SETTINGS, rng_mode="decorrelated", camera_seeds="camera", gather_passes=2, adjoint_passes=2)
    g = Renderer.from_scene(box, st)
    o = OracleRenderer(box, st, bvh_kind=0)
    try:
        full = g.render_forward()
        dl = {n: ((full[n + "_raw"][..., :3] - 0.5 * full[n + "_raw"][..., :3].mean())
                  / full[n + "_raw"][..., :3].size).astype(np.float32) for n in box.camera_names}
        g_all, _ = g.render_backward(dl)
        total = np.zeros_like(g_all["opacity"], dtype=np.float64)
        for n in box.camera_names:
            one = g.render_forward(n)
            for k in (n, n + "_raw"):
                np.testing.assert_array_equal(one[k], full[k])
            ref = o.render_forward(n)
            a, b = one[n + "_raw"][..., :3], ref[n + "_raw"][..., :3]
            assert np.median(np.abs(a - b) / np.maximum(np.abs(b), 1e-3)) < 1e-4, n
            gn, _ = g.render_backward({n: dl[n]})
            gon, _ = o.render_backward({n: dl[n]})
            x = to_asset(gn["opacity"], g.get_point_order()).astype(np.float64)
            y = to_asset(gon["opacity"], o.get_point_order()).astype(np.float64)
            cos = x @ y / (np.linalg.norm(x) * np.linalg.norm(y))
            rel = np.linalg.norm(x - y) / np.linalg.norm(y)
            assert cos >= 0.99 and rel <= 1e-2, (n, cos, rel)
            total += gn["opacity"]
        ref_all = g_all["opacity"].astype(np.float64)
        assert np.linalg.norm(total - ref_all) <= 1e-4 * np.linalg.norm(ref_all)
    finally:
        g.close()
        o.close()
