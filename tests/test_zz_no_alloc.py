"""The allocation-free LBVH build.

pale_build_lbvh_noalloc exists for callers that cannot allocate device
memory around a call (code running during CUDA-graph capture, host
applications whose own allocator owns the device memory, latency-critical
loops that cannot take cudaMalloc's implicit synchronisation).  It keeps its
temporaries in a fixed device array inside the library.  Its result must
equal the LBVH the allocating path (pale_create) builds, on two calls in a
row, and sizes above the fixed maximum must be refused with an error.

The sizes cover the single-leaf root (n <= leaf size), an ordinary build and
the fixed maximum, where every sort tile and the full scratch array are in
use.  This file is collected last so that a failure here does not hide the
results of the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from differentiablepointrendering_b200 import _native as N
from differentiablepointrendering_b200.pale import Renderer
from differentiablepointrendering_b200.scene import make_box_scene

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("n", [3, 3000, N.NOALLOC_MAX_SURFELS])
def test_noalloc_lbvh_equals_allocating_build_on_two_calls(gpu, n):
    import torch

    leaf = 4
    scene = make_box_scene(n, cameras=1, resolution=32)
    r = Renderer.from_scene(scene, {"photons": 1000, "forward_passes": 1, "gather_radius": 0.02,
                                    "leaf_size": leaf})
    codes_ref, nodes_ref = r.get_bvh()
    order_ref = r.get_point_order()
    r.close()
    lib = N.load_library()
    assert lib.pale_lbvh_node_count(n, leaf) == nodes_ref.shape[0]

    dev = torch.device("cuda:0")
    pts = scene.points
    pos = torch.from_numpy(pts["position"]).to(dev).contiguous()
    tu = torch.from_numpy(pts["tangent_u"]).to(dev).contiguous()
    tv = torch.from_numpy(pts["tangent_v"]).to(dev).contiguous()
    sc = torch.from_numpy(pts["scale"]).to(dev).contiguous()
    assert pos.shape[0] == n
    codes = torch.empty(n, dtype=torch.int32, device=dev)
    order = torch.empty(n, dtype=torch.int32, device=dev)
    nodes = torch.empty((lib.pale_lbvh_node_count(n, leaf), 16), dtype=torch.float32, device=dev)
    status = torch.empty(1, dtype=torch.int32, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    first = None
    for call in range(2):
        codes.fill_(-1)
        order.fill_(-1)
        nodes.fill_(float("nan"))
        status.fill_(-1)
        rc = lib.pale_build_lbvh_noalloc(_ptr(pos), _ptr(tu), _ptr(tv), _ptr(sc), n, leaf, _ptr(codes),
                                         _ptr(order), _ptr(nodes), _ptr(status), stream)
        torch.cuda.synchronize()
        assert rc == 0, lib.pale_last_error(None)
        assert int(status.item()) == 0, f"call {call}: device error flags"
        got = (codes.cpu().numpy().view(np.uint32), order.cpu().numpy().view(np.uint32),
               nodes.cpu().numpy().view(np.uint32))
        # integer work is compared bit-exactly, as for the allocating build
        np.testing.assert_array_equal(got[0], codes_ref, err_msg=f"call {call}")
        np.testing.assert_array_equal(got[1], order_ref, err_msg=f"call {call}")
        np.testing.assert_array_equal(got[2], nodes_ref.view(np.uint32), err_msg=f"call {call}")
        if first is None:
            first = got
        else:
            for a, b in zip(first, got):
                np.testing.assert_array_equal(a, b)


def test_noalloc_lbvh_empty_input_clears_status(gpu):
    import torch

    lib = N.load_library()
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda:0")
    rc = lib.pale_build_lbvh_noalloc(None, None, None, None, 0, 4, None, None, None, _ptr(status), None)
    torch.cuda.synchronize()
    assert rc == 0
    assert int(status.item()) == 0
    assert lib.pale_lbvh_node_count(0, 4) == 0


def test_noalloc_lbvh_rejects_sizes_above_its_maximum(gpu):
    lib = N.load_library()
    big = N.NOALLOC_MAX_SURFELS + 1
    rc = lib.pale_build_lbvh_noalloc(None, None, None, None, big, 4, None, None, None, None, None)
    assert rc == -1
    assert b"exceed the fixed maximum" in lib.pale_last_error(None)
