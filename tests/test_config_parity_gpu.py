"""Parity at the benchmarked configurations themselves.

* The mixed-size batch exactly as the bench times it: 512 uneven RGBA8 images
  (W and H log-uniform in 1..4096 plus the 1x1, 3x5, 17x13 and 4096x64 strips,
  about 20 % transparent), each with its own alpha-associated palette of 2..256
  colours, dithered in ONE call; every image's index map is compared with the
  oracle's sequential walk of that image alone (rd_riemersma_cpu.cpp:359-417),
  bit for bit.
* The 4K headline frame (RGB8, 256 colours) and a 4K RGBA8 frame with an
  alpha-associated palette, compared with the reference's own CPU build
  (oracle/_ref: RiemersmaWalkCpu compiled from the reference sources), RgbaF
  output bits against RgbaF output bits.
* The 4K block walk at the longest block of the sweep (B = 65536) against the
  oracle's RiemersmaBlocksCpu restatement, and at B = 256 against the
  reference build.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor
import os

import numpy as np
import pytest

import stipple_b200 as sb
from stipple_b200 import synth

pytestmark = pytest.mark.gpu


def test_mixed_batch_every_image_bitexact(ctx, oracle):
    spec = synth.mixed_batch_spec(512)
    imgs = [synth.gradient_rgba8(w, h, seed) for w, h, seed, _ in spec]
    pids = [ctx.palette_from_image(img, colors, associate_alpha=True)
            for img, (_, _, _, colors) in zip(imgs, spec)]
    try:
        got = ctx.dither_host("seq", imgs, pids)  # one call: the whole batch
    finally:
        for p in pids:
            ctx.release_palette(p)

    def want(i):
        w, h, _, colors = spec[i]
        idx, _, _ = oracle.walk_seq(synth.to_q16(imgs[i]), colors, True, synth.is_grayscale(imgs[i]))
        return idx

    # The oracle releases the GIL inside its C walk: spread the images over the
    # host's cores, largest first.
    order = sorted(range(len(spec)), key=lambda i: -spec[i][0] * spec[i][1])
    with ThreadPoolExecutor(max_workers=max(1, min(16, os.cpu_count() or 1))) as ex:
        wants = dict(zip(order, ex.map(want, order)))
    bad = [i for i in range(len(spec)) if not np.array_equal(got[i], wants[i])]
    assert not bad, [(i, spec[i]) for i in bad[:8]]


@pytest.mark.parametrize("alpha,colors", [(False, 256), (True, 64)])
def test_4k_sequential_against_reference_build(ctx, reflib, alpha, colors):
    img = synth.gradient_rgba8(3840, 2160, 1) if alpha else synth.gradient_rgb8(3840, 2160, 1)
    t = sb.Octree(img, colors, alpha)
    pid = ctx.palette_from_octree(t)
    try:
        _, rgba = ctx.dither_host("seq", img, pid, rgba=True)
    finally:
        ctx.release_palette(pid)
    want, _ = reflib.walk_seq(synth.to_q16(img), colors, alpha, t.grayscale)
    assert np.array_equal(rgba.view(np.uint32), want.view(np.uint32))


def test_4k_blocks_longest_block(ctx, oracle):
    img = synth.video_frame(3840, 2160, 3, 7)
    t = sb.Octree(img, 256, False)
    pid = ctx.palette_from_octree(t)
    try:
        got = ctx.dither_host("blocks", img, pid, block=65536)
    finally:
        ctx.release_palette(pid)
    want, _, _ = oracle.walk_blocks(synth.to_q16(img), 256, False, t.grayscale, 65536)
    assert np.array_equal(got, want)


def test_4k_blocks_against_reference_build(ctx, reflib):
    img = synth.video_frame(3840, 2160, 3, 0)
    t = sb.Octree(img, 256, False)
    pid = ctx.palette_from_octree(t)
    try:
        _, rgba = ctx.dither_host("blocks", img, pid, rgba=True, block=256)
    finally:
        ctx.release_palette(pid)
    want, _ = reflib.walk_blocks(synth.to_q16(img), 256, False, t.grayscale, 256)
    assert np.array_equal(rgba.view(np.uint32), want.view(np.uint32))
