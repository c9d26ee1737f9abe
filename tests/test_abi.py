"""The C-ABI library loads, exports every declared entry point, and its
host-side argument handling works without a GPU."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from differentiablepointrendering_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "pale_b200.h")).read()
    return sorted(set(re.findall(r"\b(pale_[a-z_0-9]+)\s*\(", text)))


def test_header_lists_all_python_bindings():
    assert sorted(N.EXPORTED) == declared_symbols()


def test_library_exports_every_declared_symbol():
    lib = N.load_library()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_default_settings_match_reference_defaults():
    lib = N.load_library()
    s = N.PaleSettings()
    lib.pale_default_settings(C.byref(s))
    ref = N.default_settings()
    for k, _ in N.PaleSettings._fields_:
        assert getattr(s, k) == pytest.approx(getattr(ref, k)), k
    # PathTracerSettings defaults (GPUDataStructures.h:407-422)
    assert (s.photons_per_launch, s.max_bounces, s.forward_passes, s.gather_passes) == (1000000, 6, 6, 6)
    assert (s.adjoint_bounces, s.adjoint_passes, s.rr_start, s.random_number) == (6, 6, 6, 42)
    assert (s.q_null, s.q_reflect, s.q_transmit) == (0.5, 0.5, 0.0)


def test_settings_dict_mapping():
    s = N.settings_from_dict({"photons": 1e5, "bounces": 4, "forward_passes": 2, "gather_passes": 3,
                              "adjoint_bounces": 5, "adjoint_passes": 7, "seed": 9, "logging": 4,
                              "gather_radius": 0.02, "rng_mode": "decorrelated"})
    assert (s.photons_per_launch, s.max_bounces, s.forward_passes, s.gather_passes) == (100000, 4, 2, 3)
    assert (s.adjoint_bounces, s.adjoint_passes, s.seed, s.rng_mode) == (5, 7, 9, 1)
    assert s.gather_radius == pytest.approx(0.02)
    with pytest.raises(KeyError):
        N.settings_from_dict({"no_such_key": 1})


def test_create_rejects_null_arguments_without_touching_the_gpu():
    lib = N.load_library()
    h = C.c_void_p()
    assert lib.pale_create(None, None, C.byref(h)) == -1
    assert b"null" in lib.pale_last_error(None)
    assert lib.pale_destroy(None) == 0
    assert lib.pale_point_count(None, None) == -1


def test_struct_layouts_match_header():
    # pale_settings: 6 u32, u64 (aligned at 24), 2 u32, 4 f32, 3 u32, 2 f32
    assert C.sizeof(N.PaleSettings) == 80
    assert C.sizeof(N.PalePoints) == 8 + 8 * 8
    assert N.PaleSettings.seed.offset == 24
