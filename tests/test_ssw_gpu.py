"""The speculative segmented walk (seq_mode=2): bit-exact with the reference
CPU walk for every segmentation, memo table included.  Short segments and
short warm-ups force many passes, so the verification and the pass loop are
exercised, not only the happy path."""
from __future__ import annotations

import numpy as np
import pytest

import stipple_b200 as sb
from stipple_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("alpha", [False, True])
@pytest.mark.parametrize("seg,warm", [(64, 16), (256, 64), (2048, 1024)])
def test_segmented_matches_oracle(ctx, oracle, alpha, seg, warm):
    for k, (w, h, colors) in enumerate([(256, 192, 16), (300, 211, 256), (97, 403, 64)]):
        img = synth.gradient_rgba8(w, h, 40 + k) if alpha else synth.gradient_rgb8(w, h, 40 + k)
        t = sb.Octree(img, colors, alpha)
        pid = ctx.palette_from_octree(t)
        try:
            got = ctx.dither_host("seq", img, pid, seq_mode=2, seg_len=seg, warm_len=warm)
            want, _, _ = oracle.walk_seq(synth.to_q16(img), colors, alpha, t.grayscale)
            assert np.array_equal(got, want), (w, h, colors, seg, warm)
        finally:
            ctx.release_palette(pid)


def test_segmented_no_cache_and_diffusion(ctx, oracle):
    img = synth.gradient_rgb8(400, 300, 8)
    t = sb.Octree(img, 32, False)
    pid = ctx.palette_from_octree(t)
    q = synth.to_q16(img)
    try:
        for cache in (0, 1):
            for diff in (0.5, 1.0):
                got = ctx.dither_host("seq", img, pid, seq_mode=2, seg_len=128, warm_len=32,
                                      use_cache=cache, diffusion=diff)
                want, _, _ = oracle.walk_seq(q, 32, False, False, diffusion=diff, use_cache=bool(cache))
                assert np.array_equal(got, want), (cache, diff)
    finally:
        ctx.release_palette(pid)


def test_segmented_batch_rgba_out(ctx, oracle):
    """Many uneven images in one segmented launch, RgbaF output included."""
    sizes = [(1, 1), (3, 5), (17, 13), (640, 64), (129, 257), (512, 480), (64, 64)]
    imgs, pids, want = [], [], []
    for k, (w, h) in enumerate(sizes):
        alpha = k % 2 == 1
        img = synth.gradient_rgba8(w, h, 70 + k) if alpha else synth.gradient_rgb8(w, h, 70 + k)
        colors = [16, 256, 8, 64, 2, 256, 4][k]
        t = sb.Octree(img, colors, alpha)
        pids.append(ctx.palette_from_octree(t))
        imgs.append(img)
        want.append(oracle.walk_seq(synth.to_q16(img), colors, alpha, t.grayscale))
    try:
        got, rgba = ctx.dither_host("seq", imgs, pids, rgba=True, seq_mode=2, seg_len=256,
                                    warm_len=128)
        for k in range(len(imgs)):
            assert np.array_equal(got[k], want[k][0]), sizes[k]
            _, out, _ = want[k]
            alpha = k % 2 == 1
            ch = 4 if alpha else 3
            assert np.array_equal(rgba[k][..., :ch], out[..., :ch]), sizes[k]
    finally:
        for p in pids:
            ctx.release_palette(p)


def test_segmented_full_hd(ctx, oracle):
    img = synth.gradient_rgb8(1920, 1080, 2)
    t = sb.Octree(img, 256, False)
    pid = ctx.palette_from_octree(t)
    try:
        got = ctx.dither_host("seq", img, pid, seq_mode=2)
        want, _, _ = oracle.walk_seq(synth.to_q16(img), 256, False, False)
        assert np.array_equal(got, want)
        auto = ctx.dither_host("seq", img, pid)  # automatic mode segments a 1080p frame
        assert np.array_equal(auto, want)
    finally:
        ctx.release_palette(pid)


def test_segmented_float_in_place(ctx, oracle):
    """RgbaF input is dithered in place on the device: later passes must still
    see the source pixels, so the RgbaF result is written once, at the end."""
    for alpha in (True, False):
        img = synth.gradient_rgba8(192, 160, 31) if alpha else synth.gradient_rgb8(192, 160, 31)
        q = synth.to_q16(img)
        t = sb.Octree(img, 64, alpha)
        pid = ctx.palette_from_octree(t)
        try:
            for mode in ((2, 3) if not alpha else (2,)):
                idx, rgba = ctx.dither_host("seq", q, pid, rgba=True, seq_mode=mode, seg_len=128,
                                            warm_len=32)
                want, out, _ = oracle.walk_seq(q, 64, alpha, t.grayscale)
                assert np.array_equal(idx, want), (alpha, mode)
                ch = 4 if alpha else 3
                assert np.array_equal(rgba[..., :ch].view(np.uint32), out[..., :ch].view(np.uint32))
        finally:
            ctx.release_palette(pid)
