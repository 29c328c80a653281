"""rdb_request_bytes: the device-memory bound the request loop admits by, on
the host (no GPU).  It grows with the image, counts the alpha tables and the
device palette build's scratch, and refuses a malformed request."""
from __future__ import annotations

import stipple_b200 as sb
from stipple_b200 import synth


def test_bound_grows_with_size_and_counts_what_a_request_holds():
    small = synth.gradient_rgb8(256, 256, 1)
    big = synth.gradient_rgb8(1024, 1024, 1)
    rgba = synth.gradient_rgba8(1024, 1024, 1)
    b_small = sb.Server.request_bytes(small, 64, "seq")
    b_big = sb.Server.request_bytes(big, 64, "seq")
    assert 0 < b_small < b_big
    # At least the staged input, the index map and the visit order per pixel.
    assert b_big >= 1024 * 1024 * (3 + 1 + 4)
    # Alpha: a 2^24-byte uniform-key table and hashed key maps.
    assert sb.Server.request_bytes(rgba, 64, "seq", alpha=True) > b_big + (1 << 24)
    # RgbaF output staging, 16 bytes a pixel.
    assert sb.Server.request_bytes(big, 64, "seq", rgba=True) >= b_big + 16 * 1024 * 1024
    # A palette built on the device adds its classification scratch.
    assert sb.Server.request_bytes(big, 64, "seq", device_palettes=True) > b_big


def test_engines_have_their_own_bounds():
    img = synth.gradient_rgb8(1024, 768, 2)
    seq = sb.Server.request_bytes(img, 16, "seq")
    blocks = sb.Server.request_bytes(img, 16, "blocks")
    jacobi = sb.Server.request_bytes(img, 16, "jacobi")
    # The segmented walk keeps memo tables and queues per segment; the block
    # engine a copy of the samples and indices.
    assert seq > blocks > 0 and jacobi > 0
    # Small images take the one-warp walk: one memo slab (2^18 keys, or 2^24
    # with alpha) instead of segment scratch.
    tiny = synth.gradient_rgba8(40, 40, 3)
    assert sb.Server.request_bytes(tiny, 16, "seq", alpha=True) >= (1 << 25)


def test_malformed_request_has_no_bound():
    import ctypes as C
    r = sb.Request()
    assert sb.load().rdb_request_bytes(C.byref(r), 0) == 0
    assert sb.load().rdb_request_bytes(None, 0) == 0
