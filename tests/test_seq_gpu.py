"""Sequential-exact engine on the GPU against the oracle and the golden vectors.

Bit-exact: every pixel's palette index (hence its colour) equals the
reference CPU walk's, memo table included."""
from __future__ import annotations

import numpy as np
import pytest

import golden
import stipple_b200 as sb
from stipple_b200 import synth

pytestmark = pytest.mark.gpu


def _colours(pal, idx, assoc):
    ch = 4 if assoc else 3
    return np.asarray(pal)[np.asarray(idx).reshape(-1)][:, :ch]


def _palette(ctx, tree, assoc):
    return ctx.palette(tree.palette, tree.child, tree.color_number, tree.number_unique, assoc,
                       parent=tree.parent)


@pytest.mark.parametrize("name,rgbaf,recs", list(golden.cases()),
                         ids=lambda v: v if isinstance(v, str) else "")
def test_seq_matches_golden(ctx, oracle, name, rgbaf, recs):
    for r in recs:
        colors, assoc, gray = int(r["colors"]), bool(r["assoc"]), bool(r["gray"])
        tree = oracle.build_tree(rgbaf, colors, assoc, gray)
        pid = _palette(ctx, tree, assoc)
        try:
            idx, rgba = ctx.dither_host("seq", rgbaf, pid, rgba=True)
            assert np.array_equal(_colours(r["pal"], idx, assoc), _colours(r["pal"], r["seq"], assoc)), \
                (name, colors)
            # RgbaF output: palette colour, and source alpha when alpha is not associated.
            want = np.asarray(r["pal"], np.float32)[r["seq"].reshape(-1)]
            if not assoc:
                want[:, 3] = rgbaf.reshape(-1, 4)[:, 3]
            assert np.array_equal(rgba.reshape(-1, 4), want)
            nc = ctx.dither_host("seq", rgbaf, pid, use_cache=0)
            assert np.array_equal(_colours(r["pal"], nc, assoc),
                                  _colours(r["pal"], r["seq_nocache"], assoc)), (name, colors)
        finally:
            ctx.release_palette(pid)


@pytest.mark.parametrize("alpha", [False, True])
def test_seq_matches_oracle_seeded(ctx, oracle, alpha):
    sizes = [(1, 1), (2, 1), (1, 2), (3, 5), (17, 13), (64, 64), (100, 37), (37, 100),
             (256, 192), (512, 480), (640, 64), (129, 257)]
    for k, (w, h) in enumerate(sizes):
        for colors in (2, 8, 64, 256):
            img = synth.gradient_rgba8(w, h, 11 + k) if alpha else synth.gradient_rgb8(w, h, 11 + k)
            t = sb.Octree(img, colors, alpha)
            pid = ctx.palette_from_octree(t)
            try:
                idx = ctx.dither_host("seq", img, pid)
                oidx, _, opal = oracle.walk_seq(synth.to_q16(img), colors, alpha, t.grayscale)
                assert np.array_equal(idx, oidx), (w, h, colors)
            finally:
                ctx.release_palette(pid)


def test_seq_diffusion_and_cache_options(ctx, oracle):
    img = synth.gradient_rgb8(160, 120, 5)
    t = sb.Octree(img, 32, False)
    pid = ctx.palette_from_octree(t)
    q = synth.to_q16(img)
    try:
        for diff in (0.0, 0.5, 1.0, 1.25):
            for cache in (0, 1):
                idx = ctx.dither_host("seq", img, pid, diffusion=diff, use_cache=cache)
                oidx, _, _ = oracle.walk_seq(q, 32, False, False, diffusion=diff, use_cache=bool(cache))
                assert np.array_equal(idx, oidx), (diff, cache)
        # The one-warp chain's shared-memory memo cache (the automatic mode
        # segments an image this size, which has no such cache).
        for mode in (0, 1):
            idx = ctx.dither_host("seq", img, pid, seq_mode=mode)
            assert np.array_equal(idx, oracle.walk_seq(q, 32, False, False)[0]), mode
        for bits in (4, 8, 12, 15):
            idx = ctx.dither_host("seq", img, pid, cache_bits=bits, seq_mode=1)
            oidx, _, _ = oracle.walk_seq(q, 32, False, False)
            assert np.array_equal(idx, oidx), bits
        # 2^17 entries do not fit in shared memory: refused, not truncated.
        with pytest.raises(sb.RdbError):
            ctx.dither_host("seq", img, pid, cache_bits=17, seq_mode=1)
    finally:
        ctx.release_palette(pid)


def test_seq_float_input(ctx, oracle):
    """RgbaF input (the drop-in path) with values that are not 8-bit multiples."""
    rng = np.random.default_rng(3)
    q = (rng.random((48, 72, 4)) * 65535.0).astype(np.float32)
    q[..., 3] = np.where(rng.random((48, 72)) < 0.3, q[..., 3], 65535.0)
    for alpha in (False, True):
        tree = oracle.build_tree(q, 64, alpha, False)
        pid = _palette(ctx, tree, alpha)
        try:
            idx = ctx.dither_host("seq", q, pid)
            oidx, _, _ = oracle.walk_seq(q, 64, alpha, False)
            assert np.array_equal(idx, oidx)
        finally:
            ctx.release_palette(pid)


def test_seq_batch_equals_solo(ctx, oracle):
    """Each image gives the same bytes alone and inside a batch (one launch,
    uneven sizes, mixed palettes and alpha)."""
    sizes = synth.log_uniform_sizes(40, seed=9, lo=1, hi=300) + [(1, 1), (3, 5), (17, 13), (300, 8)]
    imgs, pids, want = [], [], []
    for k, (w, h) in enumerate(sizes):
        alpha = k % 3 == 0
        colors = [2, 4, 8, 16, 64, 256][k % 6]
        img = synth.gradient_rgba8(w, h, 100 + k) if alpha else synth.gradient_rgb8(w, h, 100 + k)
        t = sb.Octree(img, colors, alpha)
        pids.append(ctx.palette_from_octree(t))
        imgs.append(img)
        want.append(oracle.walk_seq(synth.to_q16(img), colors, alpha, t.grayscale)[0])
    try:
        got = ctx.dither_host("seq", imgs, pids)
        for k in range(len(imgs)):
            assert np.array_equal(got[k], want[k]), sizes[k]
        solo = ctx.dither_host("seq", imgs[5], pids[5])
        assert np.array_equal(solo, got[5])
        again = ctx.dither_host("seq", imgs, pids)  # slabs reused: next generation
        for k in range(len(imgs)):
            assert np.array_equal(again[k], want[k])
        with pytest.raises(sb.RdbError):
            ctx.dither_host("seq", imgs[0], pids[0], cache_bits=3, seq_mode=1)
    finally:
        for p in pids:
            ctx.release_palette(p)


def test_seq_full_hd_properties(ctx, oracle):
    """1920x1080 at 256 colours: exact against the oracle, and deterministic."""
    img = synth.gradient_rgb8(1920, 1080, 2)
    t = sb.Octree(img, 256, False)
    pid = ctx.palette_from_octree(t)
    try:
        a = ctx.dither_host("seq", img, pid)
        b = ctx.dither_host("seq", img, pid)
        assert np.array_equal(a, b)
        oidx, _, _ = oracle.walk_seq(synth.to_q16(img), 256, False, False)
        assert np.array_equal(a, oidx)
    finally:
        ctx.release_palette(pid)


def test_seq_refuses_large_palette(ctx):
    img = synth.gradient_rgb8(64, 64, 1)
    t = sb.Octree(img, 1024, False)
    if t.count > 256:
        with pytest.raises(sb.RdbError):
            ctx.palette_from_octree(t)
