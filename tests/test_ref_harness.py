"""CPU checks of the reference-kernel harness (oracle/build_ref.py,
oracle/ref_harness.cu): the cited kernels are found at their cited line spans
in the reference sources, and the built library exports the harness entry
points.  The harness itself runs on the GPU (tests/test_gpu_ref_pin.py)."""
import ctypes
import os

import pytest

import build_ref
import ref as R

HAVE_SRC = os.path.isdir(os.path.join(build_ref.DEFAULT_SRC, "src", "core"))


@pytest.mark.skipif(not HAVE_SRC, reason="reference sources not present")
def test_every_cited_kernel_is_found_at_its_span():
    text = build_ref.extract(build_ref.DEFAULT_SRC)  # raises on a span mismatch
    for fname, name, lo, hi in build_ref.KERNELS:
        assert f"// ---- {fname}:{lo}-{hi}" in text
        assert name in text
    # kernels are copied whole: braces balance
    assert text.count("{") == text.count("}")


def test_harness_library_exports_its_entry_points():
    if not R.available():
        pytest.skip("oracle/_ref/libref_kernels.so not built")
    L = ctypes.CDLL(R.LIB_PATH)
    for sym in ("ref_last_error", "ref_record_fields", "ref_forward", "ref_adjoint", "ref_prox", "ref_restart_sum",
                "ref_objective", "ref_solve"):
        assert hasattr(L, sym), sym
    assert R.lib().ref_record_fields() == len(R.RECORD_FIELDS)
