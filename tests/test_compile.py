"""Compile-time contract of the C++ drop-in (the reference checks the same
with try_compile on test/bad_objectives.cu, CMakeLists.txt:291-326)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not available")
def test_objective_without_dual_overload_does_not_compile(tmp_path):
    cmd = ["nvcc", "-std=c++20", "--expt-relaxed-constexpr", "-gencode",
           "arch=compute_100a,code=sm_100a", "-I", str(ROOT / "include"), "-I",
           str(ROOT / "zeus_b200" / "csrc"), "-c", str(ROOT / "tests" / "cpp" / "bad_objective.cu"),
           "-o", str(tmp_path / "bad.o")]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode != 0
    assert "zeus::Zeus" in r.stdout + r.stderr  # no viable overload: the concept rejects it
