"""The device builders' level-synchronous decompositions (blas_build.cu, tlas_build.cu), modelled
on the CPU (tests/level_twins/level_twins.cpp) and checked against the host builders they must
reproduce word for word (host/blas.cpp, host/tlas.cpp): ranges split a binary depth at a time,
min/max reductions in shuffled order through order keys, ids and child slots from the ranges,
the top level's collapse and preorder, and both median fallbacks."""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "renderlab_b200" / "csrc"


def test_level_synchronous_builds_equal_the_host_builders(tmp_path):
    cxx = os.environ.get("CXX", "g++")
    if not shutil.which(cxx):
        pytest.skip("no C++ compiler")
    exe = tmp_path / "level_twins"
    cmd = [cxx, "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-I", str(CSRC),
           str(ROOT / "tests" / "level_twins" / "level_twins.cpp"), str(CSRC / "host" / "blas.cpp"),
           str(CSRC / "host" / "tlas.cpp"), "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, env={**os.environ, "TMPDIR": str(tmp_path)})
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mismatches 0" in r.stdout
