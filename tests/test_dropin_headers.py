"""The drop-in's headers carry the reference's header names, so objective
code written for the reference compiles unchanged: the reference's own
example programs and objective classes are compiled where they lie, against
include/ (no GPU needed to build; they run in test_gpu_reference_examples)."""
import os
from pathlib import Path

import pytest

from zeus_b200 import build as zbuild

ROOT = Path(__file__).resolve().parent.parent
REFERENCE = Path(os.environ.get("ZEUS_REFERENCE_DIR") or ROOT.parent / "reference")


def test_reference_header_names_exist():
    for h in ("zeus.cuh", "duals.cuh", "matrix.hpp", "traits.hpp"):
        assert (ROOT / "include" / h).exists(), h


@pytest.mark.skipif(not (REFERENCE / "examples" / "optimize_rosenbrock.cu").exists(),
                    reason="reference checkout not present")
def test_reference_examples_compile_against_include():
    bins = zbuild.build_reference_examples(REFERENCE)
    assert {b.name for b in bins} == set(zbuild.REF_PROGRAMS)
    for b in bins:
        assert b.exists() and os.access(b, os.X_OK)
    # the relative include of optimization_utils.hpp reaches this library's
    # traits.hpp, not the reference's
    tree = zbuild.BUILD / "ref_examples"
    assert (tree / "examples" / ".." / "include" / "traits.hpp").resolve() == \
        (ROOT / "include" / "traits.hpp").resolve()
