"""The build's extra nvcc flags (PALE_NVCC_FLAGS): a changed flag set
rebuilds the library and is recorded beside it; an unchanged one with
up-to-date sources does not rebuild.  nvcc is replaced by a stub that
writes the output file, so nothing is compiled."""
import os
import shutil

import pytest

import differentiablepointrendering_b200.build as B


@pytest.fixture
def pkg(tmp_path, monkeypatch):
    # a copy of the package's sources and header in a scratch tree
    here = os.path.dirname(B.__file__)
    root = tmp_path / "repo"
    pk = root / "pkg"
    shutil.copytree(os.path.join(here, "csrc"), pk / "csrc")
    (root / "include").mkdir(parents=True)
    shutil.copy(os.path.join(here, "..", "include", "pale_b200.h"), root / "include")
    monkeypatch.setattr(B, "HERE", str(pk))
    monkeypatch.setattr(B, "nvcc", lambda: "nvcc")
    calls = []

    def run(cmd, check):
        calls.append(cmd)
        out = cmd[cmd.index("-o") + 1]
        with open(out, "w") as f:
            f.write("lib")

    monkeypatch.setattr(B.subprocess, "run", run)
    return pk, calls


def test_flags_rebuild_and_stamp(pkg, monkeypatch):
    pk, calls = pkg
    monkeypatch.delenv("PALE_NVCC_FLAGS", raising=False)
    out = B.build_library()
    assert len(calls) == 1 and os.path.exists(out)
    assert open(out + ".flags").read() == ""
    B.build_library()
    assert len(calls) == 1                      # sources and flags unchanged
    monkeypatch.setenv("PALE_NVCC_FLAGS", "-DPALE_REFILL_STEPS=32 -DPALE_ROUND_MIN_BLOCKS=4")
    B.build_library()
    assert len(calls) == 2
    assert "-DPALE_REFILL_STEPS=32" in calls[-1] and "-DPALE_ROUND_MIN_BLOCKS=4" in calls[-1]
    assert "-fmad=false" in calls[-1]           # the parity flags stay
    assert open(out + ".flags").read() == "-DPALE_REFILL_STEPS=32 -DPALE_ROUND_MIN_BLOCKS=4"
    B.build_library()
    assert len(calls) == 2
    monkeypatch.delenv("PALE_NVCC_FLAGS")
    B.build_library()
    assert len(calls) == 3 and "-DPALE_REFILL_STEPS=32" not in calls[-1]
