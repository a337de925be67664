"""Host-side view-set bookkeeping, on the CPU: where each view's pixels sit
in a set's concatenated image (the library's set_views places them)."""
from tensorray_b200 import api
from tensorray_b200._abi import TrnView


def _views(specs):
    arr = (TrnView * len(specs))()
    for i, (w, h, off) in enumerate(specs):
        arr[i].camera.width, arr[i].camera.height, arr[i].pixel_offset = w, h, off
    return arr


def test_views_without_offsets_are_packed():
    assert api.ViewSet._offsets(_views([(4, 2, -1), (3, 3, -1), (2, 2, -1)]), 3) == [0, 8, 17]


def test_explicit_offsets_are_kept_and_the_next_view_follows():
    assert api.ViewSet._offsets(_views([(4, 2, -1), (2, 2, 100), (1, 1, -1)]), 3) == [0, 100, 104]
    # two views may share pixels (accumulate into one image)
    assert api.ViewSet._offsets(_views([(4, 2, 0), (4, 2, 0), (1, 1, -1)]), 3) == [0, 0, 8]
