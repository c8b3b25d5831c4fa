"""The Allen adaptor's view structs against the reference's own view types, on the host (no GPU):
tests/allen_harness builds the reference's Hits, Track, Tracks and MultiEventTracks with their own
constructors and compares them byte for byte with include/velo_b200.h's structs filled as
velo_create_velo_views fills them."""
import ctypes as C
import os

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HARNESS = os.path.join(REPO, "tests", "allen_harness", "_build", "libvelo_allen_harness.so")


@pytest.mark.skipif(not os.path.exists(HARNESS), reason="Allen harness not built (needs the reference tree)")
def test_view_layouts_equal_the_reference_types():
    lib = C.CDLL(HARNESS)
    assert lib.allen_harness_layout_check() == 0
