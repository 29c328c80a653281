"""The segmented walk on thread walkers (seq_mode=3): bit-exact with the
reference CPU walk for every segmentation, memo table included.  Short
segments and warm-ups force many passes, so the three checks and the pass
loop are exercised, not only the first pass."""
from __future__ import annotations

import numpy as np
import pytest

import stipple_b200 as sb
from stipple_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("seg,warm", [(64, 16), (256, 128), (1024, 512)])
def test_thread_segmented_matches_oracle(ctx, oracle, seg, warm, form):
    for k, (w, h, colors) in enumerate([(256, 192, 16), (300, 211, 256), (97, 403, 64)]):
        img = synth.gradient_rgb8(w, h, 40 + k)
        t = sb.Octree(img, colors, False)
        pid = ctx.palette_from_octree(t)
        try:
            got = ctx.dither_host("seq", img, pid, seq_mode=3, seg_len=seg, warm_len=warm,
                                  walk_form=form)
            want, _, _ = oracle.walk_seq(synth.to_q16(img), colors, False, t.grayscale)
            assert np.array_equal(got, want), (w, h, colors, seg, warm, form)
            assert ctx.last_passes >= 1
        finally:
            ctx.release_palette(pid)


@pytest.mark.parametrize("form", [1, 2])
def test_thread_segmented_no_cache_and_diffusion(ctx, oracle, form):
    img = synth.gradient_rgb8(400, 300, 8)
    t = sb.Octree(img, 32, False)
    pid = ctx.palette_from_octree(t)
    q = synth.to_q16(img)
    try:
        for cache in (0, 1):
            for diff in (0.5, 1.0):
                got = ctx.dither_host("seq", img, pid, seq_mode=3, seg_len=128, warm_len=32,
                                      use_cache=cache, diffusion=diff, walk_form=form)
                want, _, _ = oracle.walk_seq(q, 32, False, False, diffusion=diff, use_cache=bool(cache))
                assert np.array_equal(got, want), (cache, diff)
    finally:
        ctx.release_palette(pid)


@pytest.mark.parametrize("form", [1, 2])
def test_thread_segmented_gray_and_float(ctx, oracle, form):
    """A greyscale palette (the deepest tree, whose descent reads bits below the
    memo key) and RgbaF input that is not 8-bit multiples."""
    img = synth.gradient_rgb8(320, 200, 12)
    g = img[..., :1].repeat(3, axis=2).copy()
    t = sb.Octree(g, 16, False)
    assert t.grayscale
    pid = ctx.palette_from_octree(t)
    try:
        got = ctx.dither_host("seq", g, pid, seq_mode=3, seg_len=128, warm_len=64, walk_form=form)
        want, _, _ = oracle.walk_seq(synth.to_q16(g), 16, False, True)
        assert np.array_equal(got, want)
    finally:
        ctx.release_palette(pid)
    rng = np.random.default_rng(3)
    q = (rng.random((150, 190, 4)) * 65535.0).astype(np.float32)
    q[..., 3] = 65535.0
    tree = oracle.build_tree(q, 64, False, False)
    pid = ctx.palette(tree.palette, tree.child, tree.color_number, tree.number_unique, False,
                      parent=tree.parent)
    try:
        got = ctx.dither_host("seq", q, pid, seq_mode=3, seg_len=256, warm_len=64, walk_form=form)
        want, _, _ = oracle.walk_seq(q, 64, False, False)
        assert np.array_equal(got, want)
    finally:
        ctx.release_palette(pid)


def test_thread_segmented_batch_rgba_out(ctx, oracle):
    """Uneven images in one call, RgbaF output included; each image is the
    same as alone."""
    sizes = [(1, 1), (3, 5), (17, 13), (640, 64), (129, 257), (512, 480), (64, 64)]
    imgs, pids, want = [], [], []
    for k, (w, h) in enumerate(sizes):
        img = synth.gradient_rgb8(w, h, 70 + k) if k % 2 else synth.gradient_rgba8(w, h, 70 + k)
        colors = [16, 256, 8, 64, 2, 256, 4][k]
        t = sb.Octree(img, colors, False)
        pids.append(ctx.palette_from_octree(t))
        imgs.append(img)
        want.append(oracle.walk_seq(synth.to_q16(img), colors, False, t.grayscale))
    try:
        got, rgba = ctx.dither_host("seq", imgs, pids, rgba=True, seq_mode=3, seg_len=128,
                                    warm_len=64)
        for k in range(len(imgs)):
            assert np.array_equal(got[k], want[k][0]), sizes[k]
            _, out, _ = want[k]
            assert np.array_equal(rgba[k][..., :3], out[..., :3]), sizes[k]
            solo = ctx.dither_host("seq", imgs[k], pids[k], seq_mode=3, seg_len=128, warm_len=64)
            assert np.array_equal(solo, got[k]), sizes[k]
    finally:
        for p in pids:
            ctx.release_palette(p)


def test_thread_segmented_full_hd_auto(ctx, oracle):
    img = synth.gradient_rgb8(1920, 1080, 2)
    t = sb.Octree(img, 256, False)
    pid = ctx.palette_from_octree(t)
    try:
        want, _, _ = oracle.walk_seq(synth.to_q16(img), 256, False, False)
        got = ctx.dither_host("seq", img, pid)  # automatic mode: thread walkers for RGB
        assert np.array_equal(got, want)
        assert ctx.last_passes >= 1
    finally:
        ctx.release_palette(pid)


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("seg,warm", [(64, 16), (256, 64)])
def test_thread_segmented_alpha(ctx, oracle, seg, warm, form):
    """Alpha-associated palettes: four channels, 24-bit keys in hashed maps."""
    for k, (w, h, colors) in enumerate([(256, 192, 16), (300, 211, 256), (97, 403, 4), (640, 64, 64)]):
        img = synth.gradient_rgba8(w, h, 60 + k)
        t = sb.Octree(img, colors, True)
        pid = ctx.palette_from_octree(t)
        try:
            got, rgba = ctx.dither_host("seq", img, pid, rgba=True, seq_mode=3, seg_len=seg,
                                        warm_len=warm, walk_form=form)
            want, out, _ = oracle.walk_seq(synth.to_q16(img), colors, True, t.grayscale)
            assert np.array_equal(got, want), (w, h, colors, seg, warm)
            assert np.array_equal(rgba.view(np.uint32), out.view(np.uint32)), (w, h, colors)
        finally:
            ctx.release_palette(pid)


def test_thread_segmented_alpha_float_and_no_cache(ctx, oracle):
    rng = np.random.default_rng(5)
    q = (rng.random((120, 170, 4)) * 65535.0).astype(np.float32)
    q[..., 3] = np.where(rng.random((120, 170)) < 0.3, q[..., 3], 65535.0)
    tree = oracle.build_tree(q, 64, True, False)
    pid = ctx.palette(tree.palette, tree.child, tree.color_number, tree.number_unique, True,
                      parent=tree.parent)
    try:
        for cache in (1, 0):
            got = ctx.dither_host("seq", q, pid, seq_mode=3, seg_len=128, warm_len=32,
                                  use_cache=cache)
            want, _, _ = oracle.walk_seq(q, 64, True, False, use_cache=bool(cache))
            assert np.array_equal(got, want), cache
    finally:
        ctx.release_palette(pid)


def test_thread_segmented_mixed_alpha_batch(ctx, oracle):
    """A batch mixing alpha and plain palettes (split into one launch of each
    kind), every image equal to the oracle."""
    sizes = [(200, 100), (130, 140), (512, 64), (90, 300), (256, 256)]
    imgs, pids, want = [], [], []
    for k, (w, h) in enumerate(sizes):
        alpha = k % 2 == 0
        img = synth.gradient_rgba8(w, h, 80 + k) if alpha else synth.gradient_rgb8(w, h, 80 + k)
        colors = [256, 16, 64, 8, 128][k]
        t = sb.Octree(img, colors, alpha)
        pids.append(ctx.palette_from_octree(t))
        imgs.append(img)
        want.append(oracle.walk_seq(synth.to_q16(img), colors, alpha, t.grayscale)[0])
    try:
        got = ctx.dither_host("seq", imgs, pids, seq_mode=3, seg_len=96, warm_len=32)
        for k in range(len(imgs)):
            assert np.array_equal(got[k], want[k]), sizes[k]
        auto = ctx.dither_host("seq", imgs, pids)
        for k in range(len(imgs)):
            assert np.array_equal(auto[k], want[k]), sizes[k]
    finally:
        for p in pids:
            ctx.release_palette(p)


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("alpha", [False, True])
def test_host_and_device_pass_loops_agree(ctx, oracle, alpha, form):
    """The pass loop checked by the host (loop_mode=1) and the device-side loop
    in one CUDA graph (loop_mode=2) give the oracle's bytes; the device loop's
    pass limit surfaces as an error, never as an inexact result."""
    img = synth.gradient_rgba8(480, 320, 9) if alpha else synth.gradient_rgb8(480, 320, 9)
    t = sb.Octree(img, 64, alpha)
    pid = ctx.palette_from_octree(t)
    try:
        want, _, _ = oracle.walk_seq(synth.to_q16(img), 64, alpha, t.grayscale)
        for mode in (1, 2, 2):  # the second device-loop call reuses the cached graph
            got = ctx.dither_host("seq", img, pid, seq_mode=3, seg_len=64, warm_len=16, loop_mode=mode,
                                  walk_form=form)
            assert np.array_equal(got, want), mode
            assert ctx.last_passes >= 3
        with pytest.raises(sb.RdbError):
            ctx.dither_host("seq", img, pid, seq_mode=3, seg_len=64, warm_len=16, loop_mode=2,
                            max_passes=3)
        got = ctx.dither_host("seq", img, pid, seq_mode=3, seg_len=64, warm_len=16, loop_mode=2)
        assert np.array_equal(got, want)  # the context recovers after the error
    finally:
        ctx.release_palette(pid)


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("alpha", [False, True])
@pytest.mark.parametrize("window,seg", [(1, 32), (5, 32), (37, 48), (130, 64)])
def test_thread_segmented_window(ctx, oracle, alpha, window, seg, form):
    """One image walked a window of segments beyond the front each pass:
    segments entering the window start from warm-ups, the front stops at the
    window's end; both pass loops, with and without the memo table."""
    img = synth.gradient_rgba8(300, 170, 90) if alpha else synth.gradient_rgb8(300, 170, 90)
    t = sb.Octree(img, 64, alpha)
    pid = ctx.palette_from_octree(t)
    q = synth.to_q16(img)
    try:
        for cache in (1, 0):
            want, _, _ = oracle.walk_seq(q, 64, alpha, t.grayscale, use_cache=bool(cache))
            for mode in (1, 2):
                got = ctx.dither_host("seq", img, pid, seq_mode=3, seg_len=seg, warm_len=16,
                                      seg_window=window, use_cache=cache, loop_mode=mode,
                                      walk_form=form)
                assert np.array_equal(got, want), (cache, mode)
                # The front advances at most a window per pass.
                passes = ctx.last_passes
                print(f"window {window} seg {seg} alpha {alpha} form {form} cache {cache} "
                      f"mode {mode}: {passes} passes")
                assert passes >= -(-(300 * 170) // (seg * window)), (cache, mode, passes)
    finally:
        ctx.release_palette(pid)


def test_thread_segmented_window_float(ctx, oracle):
    rng = np.random.default_rng(6)
    q = (rng.random((90, 140, 4)) * 65535.0).astype(np.float32)
    tree = oracle.build_tree(q, 32, True, False)
    pid = ctx.palette(tree.palette, tree.child, tree.color_number, tree.number_unique, True,
                      parent=tree.parent)
    try:
        want, _, _ = oracle.walk_seq(q, 32, True, False)
        got = ctx.dither_host("seq", q, pid, seq_mode=3, seg_len=32, warm_len=16, seg_window=9)
        assert np.array_equal(got, want)
    finally:
        ctx.release_palette(pid)


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("window", [3, 40, 0, -1])
def test_thread_segmented_batch_windows(ctx, oracle, window, form):
    """Several images in one call, each walking its own window of segments
    past its front, the windows re-shared after every pass by the segments
    each image has left (window: the total shared out, at least 256 each;
    0: twice the device's resident segments; -1: no windows); both pass
    loops."""
    sizes = [(300, 170), (64, 140), (511, 97), (128, 128), (97, 61)]
    imgs, pids, want = [], [], []
    for k, (w, h) in enumerate(sizes):
        img = synth.gradient_rgb8(w, h, 120 + k)
        t = sb.Octree(img, [64, 16, 256, 8, 32][k], False)
        pids.append(ctx.palette_from_octree(t))
        imgs.append(img)
        want.append(oracle.walk_seq(synth.to_q16(img), [64, 16, 256, 8, 32][k], False, t.grayscale)[0])
    try:
        for mode in (1, 2):
            got = ctx.dither_host("seq", imgs, pids, seq_mode=3, seg_len=32, warm_len=16,
                                  seg_window=window, loop_mode=mode, walk_form=form)
            for k in range(len(imgs)):
                assert np.array_equal(got[k], want[k]), (sizes[k], mode)
    finally:
        for p in pids:
            ctx.release_palette(p)


def test_profiled_walk_reports_its_work(ctx, oracle):
    """With profiling on, the walk's statistics: one walk launch per pass,
    every image position walked at least once (counted on the device), the
    segment length asked for."""
    img = synth.gradient_rgb8(400, 300, 14)
    t = sb.Octree(img, 64, False)
    pid = ctx.palette_from_octree(t)
    try:
        want, _, _ = oracle.walk_seq(synth.to_q16(img), 64, False, t.grayscale)
        for form in (1, 2):
            ctx.profile(True)
            try:
                got = ctx.dither_host("seq", img, pid, seq_mode=3, seg_len=48, warm_len=16,
                                      seg_window=300, walk_form=form, loop_mode=1)
                k = ctx.stats()
            finally:
                ctx.profile(False)
            assert np.array_equal(got, want), form
            assert k["passes"] == ctx.last_passes == k["walk_launches"]
            assert k["seg_len"] == 48
            assert k["walk_positions"] >= 400 * 300
            assert k["walk_ms"] > 0
    finally:
        ctx.release_palette(pid)
