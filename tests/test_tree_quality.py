"""Traversal work per ray on the reference's median-split BVH (leaf size 4,
BasicBVH::buildFromBoxes, BVH.ixx:49-133, as the oracle restates it)
against the LBVH this build traverses (leaf size 1, the oracle's bit-exact
restatement of the CUDA build), on the same rays through the box200k cloud.
The kernels' algorithmic bytes count this build's own node visits and
surfel tests (32 B per node, 52 B per surfel test); this test measures them
beside the reference tree's on the same rays, and checks that both trees
find the same closest hits."""
import numpy as np

from differentiablepointrendering_b200.scene import make_box_scene, make_surfels
from oracle_lib import OracleRenderer

N_SURFELS = 200000


def _rays(n=20000):
    rng = np.random.default_rng(7)
    # from inside the cloud's box, and from a sphere around it towards it
    o_in = rng.uniform(-0.45, 0.45, (n, 3))
    d_in = rng.normal(size=(n, 3))
    u = rng.normal(size=(n, 3))
    o_out = 1.5 * u / np.linalg.norm(u, axis=1, keepdims=True)
    d_out = rng.uniform(-0.3, 0.3, (n, 3)) - o_out
    o = np.concatenate([o_in, o_out]).astype(np.float32)
    d = np.concatenate([d_in, d_out])
    return o, (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)


def test_lbvh_work_against_the_reference_tree(capsys):
    scene = make_box_scene(N_SURFELS, cameras=1, resolution=8, points=make_surfels(N_SURFELS, 1234))
    o, d = _rays()
    work, hits = {}, {}
    for kind, name in ((0, "median split, leaf 4"), (1, "LBVH, leaf 1")):
        r = OracleRenderer(scene, {"photons": 1, "forward_passes": 1, "leaf_size": 1}, bvh_kind=kind)
        inst, prim, t, _, _ = r.trace_rays(o, d)
        st = r.stats()
        n = o.shape[0]
        work[name] = (st["node_visits"] / n, st["surfel_tests"] / n)
        surf = inst == scene.instance_mesh.shape[0]
        ids = np.full(n, -1, np.int64)
        ids[surf] = r.get_point_order()[prim[surf]]
        hits[name] = (inst, ids, t)
    (ia, sa, ta), (ib, sb, tb) = hits.values()
    # the closest hit does not depend on the tree
    assert np.mean(ia == ib) > 0.9995
    assert np.mean(sa == sb) > 0.9995
    same = (ia == ib) & (ia >= 0)
    np.testing.assert_allclose(ta[same], tb[same], rtol=1e-6, atol=1e-7)
    ref_bytes = 32 * work["median split, leaf 4"][0] + 52 * work["median split, leaf 4"][1]
    our_bytes = 32 * work["LBVH, leaf 1"][0] + 52 * work["LBVH, leaf 1"][1]
    with capsys.disabled():
        for name, (nv, ts) in work.items():
            print(f"\n{name}: {nv:.1f} node visits, {ts:.1f} surfel tests, {32 * nv + 52 * ts:.0f} B per ray")
    # the LBVH's traversal bytes stay within a small factor of the reference tree's
    assert 0.3 * ref_bytes < our_bytes < 2.0 * ref_bytes
