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


def test_struct_layouts_match_header(tmp_path):
    """The ctypes structs equal the header's: a C program compiled against
    include/pale_b200.h prints the size and every field offset."""
    import shutil
    import subprocess

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    structs = {"pale_settings": N.PaleSettings, "pale_points": N.PalePoints, "pale_stats": N.PaleStats,
               "pale_scene_desc": N.PaleSceneDesc, "pale_optimizer": N.PaleOptimizer}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "pale_b200.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in cls._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, cls in structs.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for f, _ in cls._fields_:
            assert got[(cname, f)] == getattr(cls, f).offset, (cname, f)
