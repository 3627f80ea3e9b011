"""Property checks of the oracle's offset encoding (isect_offset_encode,
restating isect_tiles.cu:309-355): for sorted intersection keys
(camera << (32 + tile_bits) | tile << 32 | depth bits), offsets[c, t] is the
first intersection whose (camera, tile) index is >= c * n_tiles + t -- a
lower-bound search -- bit-exact for empty input, empty trailing tiles and
cameras without intersections.  Depth bits are those of positive floats
(every intersected splat lies beyond the near plane), so the sign extension
of the reference's key leaves the camera and tile fields intact.
"""
import numpy as np
from hypothesis import given, settings
from hypothesis import strategies as st

from oracle import oracle as O


@st.composite
def keys_case(draw):
    C = draw(st.integers(1, 4))
    tw, th = draw(st.integers(1, 9)), draw(st.integers(1, 9))
    n_tiles = tw * th
    n = draw(st.integers(0, 200))
    cams = draw(st.lists(st.integers(0, C - 1), min_size=n, max_size=n))
    tiles = draw(st.lists(st.integers(0, n_tiles - 1), min_size=n, max_size=n))
    depth_bits = draw(st.lists(st.integers(0, 2**31 - 1), min_size=n, max_size=n))
    return C, tw, th, np.array(cams, np.int64), np.array(tiles, np.int64), np.array(depth_bits, np.int64)


@settings(max_examples=150, deadline=None)
@given(keys_case())
def test_offsets_are_lower_bounds_of_the_sorted_ids(case):
    C, tw, th, cams, tiles, depth = case
    n_tiles = tw * th
    tb = O.tile_bits(n_tiles)
    keys = (cams << (32 + tb)) | (tiles << 32) | depth  # camera and tile above bit 32, depth bits below
    sorted_keys = np.sort(keys, kind="stable")
    offsets = O.isect_offset_encode(sorted_keys, C, tw, th)
    # the (camera, tile) index each sorted key decodes to, as the encoder reads it (key >> 32)
    hi = sorted_keys >> 32
    dec = (hi >> tb) * n_tiles + (hi & ((1 << tb) - 1))
    expect = np.searchsorted(dec, np.arange(C * n_tiles), side="left").astype(np.int32)
    assert offsets.shape == (C, th, tw)
    np.testing.assert_array_equal(offsets.reshape(-1), expect)
