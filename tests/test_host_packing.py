"""Host-side packing of per-camera images (pale.Renderer's forward-with-loss
and backward paths): the packed buffers and per-camera views equal what
per-camera copies and a concatenation give, bit for bit."""
import numpy as np

from differentiablepointrendering_b200.pale import _pack_rgba, _split_rgba


def test_pack_rgba_equals_padded_concatenation():
    rng = np.random.default_rng(5)
    shapes = [(4, 6), (3, 5), (7, 2)]
    rgbs = [rng.normal(size=(h, w, 3)).astype(np.float32) for h, w in shapes]
    rgbs[1] = np.asfortranarray(rgbs[1])          # any memory order in
    buf, views = _pack_rgba(rgbs)
    old = []
    for a in rgbs:
        rgba = np.ones(a.shape[:2] + (4,), np.float32)
        rgba[..., :3] = a
        old.append(rgba)
    want = np.concatenate([o.reshape(-1) for o in old])
    assert buf.dtype == np.float32 and buf.flags.c_contiguous
    np.testing.assert_array_equal(buf.view(np.uint32), want.view(np.uint32))
    for v, o in zip(views, old):
        assert v.shape == o.shape and v.base is buf
        np.testing.assert_array_equal(v, o)
    assert sum(v.size for v in views) == buf.size


def test_pack_rgba_without_images():
    buf, views = _pack_rgba([])
    assert views == [] and buf.shape == (4,) and not buf.any()


def test_split_rgba_views_match_slices():
    sizes = [(6, 4), (5, 3), (2, 7)]                  # (W, H)
    n = sum(w * h * 4 for w, h in sizes)
    buf = np.arange(n, dtype=np.float32)
    views = _split_rgba(buf, sizes)
    off = 0
    for (w, h), v in zip(sizes, views):
        np.testing.assert_array_equal(v, buf[off:off + w * h * 4].reshape(h, w, 4))
        assert v.shape == (h, w, 4) and v.flags.c_contiguous
        off += w * h * 4
    # the loss path's dL/dI: RGB of the packed float4 per pixel, contiguous
    d3 = np.ascontiguousarray(views[0][..., :3])
    np.testing.assert_array_equal(d3, buf[: 6 * 4 * 4].reshape(4, 6, 4)[..., :3])
    assert d3.flags.c_contiguous
