"""The configurations' full sizes, bit for bit against the oracle: a 3840x2160
RGB8 frame at 256 colours (the headline walk), a 3840x2160 RGBA8 frame with an
alpha-associated palette (the batched and served alpha path at its largest),
and a 3840x2160 video frame through the block engine at B = 256.  Each also
checks determinism (a second run gives the same bytes)."""
from __future__ import annotations

import numpy as np
import pytest

import stipple_b200 as sb
from stipple_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("alpha,colors", [(False, 256), (True, 64)])
def test_4k_sequential(ctx, oracle, alpha, colors):
    img = synth.gradient_rgba8(3840, 2160, 1) if alpha else synth.gradient_rgb8(3840, 2160, 1)
    t = sb.Octree(img, colors, alpha)
    pid = ctx.palette_from_octree(t)
    try:
        a = ctx.dither_host("seq", img, pid)
        b = ctx.dither_host("seq", img, pid)
        assert np.array_equal(a, b)
        want, _, _ = oracle.walk_seq(synth.to_q16(img), colors, alpha, t.grayscale)
        assert np.array_equal(a, want)
        assert ctx.last_passes >= 1
    finally:
        ctx.release_palette(pid)


def test_4k_blocks(ctx, oracle):
    img = synth.video_frame(3840, 2160, 3, 0)
    t = sb.Octree(img, 256, False)
    pid = ctx.palette_from_octree(t)
    try:
        got = ctx.dither_host("blocks", img, pid, block=256)
        want, _, _ = oracle.walk_blocks(synth.to_q16(img), 256, False, t.grayscale, 256)
        assert np.array_equal(got, want)
    finally:
        ctx.release_palette(pid)
