"""The allocation-free sequential walk (rdb_dither_seq_noalloc).

That entry point serves callers that may not allocate device memory -- for
example a plugin whose host application owns all GPU memory through its own
allocator, or a latency-critical path that cannot afford cudaMalloc's implicit
synchronisation.  It keeps its scratch in a fixed device array inside the
library.  This test calls it through the C ABI twice in a row and checks both
results against the ordinary entry point (rdb_dither), bit for bit, which is
the tolerance every test of the exact engine uses.  It is collected last and
passes alone in a fresh process as well as after the other tests.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import stipple_b200 as sb
from stipple_b200 import synth

pytestmark = pytest.mark.gpu


def _plan(tree: sb.Octree) -> bytes:
    child, parent, cn, nu = tree.nodes()
    return sb.plan_blob(tree.colormap(), child, cn, nu, False, parent=parent)


def test_noalloc_matches_rdb_dither_twice(lib):
    import torch
    if sb.device_count() < 1:
        pytest.fail("no CUDA device")
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    ctx = sb.Context(0)
    try:
        cases = [(320, 200, 64, 1), (257, 129, 256, 2)]
        for w, h, colors, seed in cases:
            img = synth.gradient_rgb8(w, h, seed)
            tree = sb.Octree(img, colors, False)
            pid = ctx.palette_from_octree(tree)
            want = ctx.dither_host("seq", img, pid)
            ctx.release_palette(pid)
            blob = np.frombuffer(_plan(tree), np.uint8).copy()
            d_img = torch.from_numpy(img).cuda()
            for call in range(2):
                d_idx = torch.full((h, w), 7, dtype=torch.uint8, device="cuda")
                # The fill above ran on torch's current stream; the walk runs on
                # `stream`, so order the two.
                stream.wait_stream(torch.cuda.current_stream())
                rc = lib.rdb_dither_seq_noalloc(blob.ctypes.data, blob.size, d_img.data_ptr(), 0,
                                                w, h, sb.RGB8, d_idx.data_ptr(), 1.0, 1,
                                                C.c_void_p(stream.cuda_stream))
                assert rc == 0, lib.rdb_last_error().decode()
                stream.synchronize()
                got = d_idx.cpu().numpy()
                assert np.array_equal(got, want), (w, h, colors, call)
    finally:
        ctx.close()


def test_noalloc_generation_wrap(lib):
    """The memo table in the shared array is told apart between calls by an
    8-bit generation that wraps after 255 calls, when the table is cleared.
    Enough calls on a small image to pass the wrap; the last ones are checked
    bit for bit against rdb_dither."""
    import torch
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    ctx = sb.Context(0)
    try:
        w, h = 16, 16
        img = synth.gradient_rgb8(w, h, 11)
        tree = sb.Octree(img, 16, False)
        pid = ctx.palette_from_octree(tree)
        want = ctx.dither_host("seq", img, pid)
        ctx.release_palette(pid)
        blob = np.frombuffer(_plan(tree), np.uint8).copy()
        d_img = torch.from_numpy(img).cuda()
        d_idx = torch.full((h, w), 7, dtype=torch.uint8, device="cuda")
        stream.wait_stream(torch.cuda.current_stream())
        for call in range(262):
            rc = lib.rdb_dither_seq_noalloc(blob.ctypes.data, blob.size, d_img.data_ptr(), 0,
                                            w, h, sb.RGB8, d_idx.data_ptr(), 1.0, 1,
                                            C.c_void_p(stream.cuda_stream))
            assert rc == 0, lib.rdb_last_error().decode()
            if call >= 250:
                stream.synchronize()
                assert np.array_equal(d_idx.cpu().numpy(), want), call
    finally:
        ctx.close()


def test_noalloc_refuses_oversized_and_alpha(lib):
    import torch
    img = synth.gradient_rgb8(64, 64, 3)
    tree = sb.Octree(img, 16, False)
    blob = np.frombuffer(_plan(tree), np.uint8).copy()
    d_idx = torch.empty(16, dtype=torch.uint8, device="cuda")
    rc = lib.rdb_dither_seq_noalloc(blob.ctypes.data, blob.size, d_idx.data_ptr(), 0,
                                    2048, 1024, sb.RGB8, d_idx.data_ptr(), 1.0, 1, None)
    assert rc == 4  # RDB_E_UNSUPPORTED
    assert b"1048576" in lib.rdb_last_error()
    imga = synth.gradient_rgba8(32, 32, 3)
    ta = sb.Octree(imga, 16, True)
    child, parent, cn, nu = ta.nodes()
    blob_a = np.frombuffer(sb.plan_blob(ta.colormap(), child, cn, nu, True, parent=parent),
                           np.uint8).copy()
    rc = lib.rdb_dither_seq_noalloc(blob_a.ctypes.data, blob_a.size, d_idx.data_ptr(), 0,
                                    4, 4, sb.RGBA8, d_idx.data_ptr(), 1.0, 1, None)
    assert rc != 0 and b"alpha" in lib.rdb_last_error()
