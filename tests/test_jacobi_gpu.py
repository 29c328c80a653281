"""The approximation engine (RDB_ENGINE_JACOBI).

Default form, block sweeps: the block-mode list in blocks of 256, all walked in
parallel and cache-free, each from its predecessor's end queue of the previous
sweep, stopping at the first sweep that changes no block's end queue.  From
then on the result is exactly the cache-free walk along the block-mode list --
the reference's block walk with the whole list as one block
(src/rd_riemersma_cpu.cpp:477-805) -- which these tests check bit for bit at
the served sizes, for every colour count of the served mix and with alpha.

Against the memoised sequential walk (the reference's RiemersmaWalkCpu with
its memo table) no order-free scheme can match: the memo answers a key with
the index its FIRST target received, a property of the order.  The measured
floor of the cache-free walk against the memoised one is the stated tolerance
(index mismatch fraction, mean CIE dE76), measured on the 1024x1024
gradient+noise workload of seed 31.

Second form (jacobi_form 1): the reference's own order-free point iteration
with the truncated inverse filter (src/rd_approx_cuda.cu), held to its stated
tolerance on a 320x240 workload."""
from __future__ import annotations

import numpy as np
import pytest

import stipple_b200 as sb
from stipple_b200 import metrics, synth

pytestmark = pytest.mark.gpu

# Block sweeps against the memoised walk: (colours, alpha) -> (max index
# mismatch, max mean dE76).  Measured: 2.45 % / 1.91, 5.01 % / 3.01,
# 6.41 % / 3.28, 5.71 % / 2.49, 5.47 % / 1.40, 6.97 % / 1.07; with alpha
# 1.42 % / 1.11, 4.07 % / 1.79, 3.89 % / 0.98.
MEMO_FLOOR = {
    (2, False): (0.030, 2.1),
    (4, False): (0.055, 3.2),
    (8, False): (0.070, 3.5),
    (16, False): (0.062, 2.7),
    (64, False): (0.060, 1.5),
    (256, False): (0.075, 1.2),
    (4, True): (0.020, 1.3),
    (16, True): (0.045, 2.0),
    (64, True): (0.045, 1.1),
}


def _image(w, h, alpha, seed):
    return synth.gradient_rgba8(w, h, seed) if alpha else synth.gradient_rgb8(w, h, seed)


@pytest.mark.parametrize("colors,alpha", list(MEMO_FLOOR))
def test_block_sweeps_reach_the_cache_free_walk(ctx, oracle, colors, alpha):
    img = _image(1024, 1024, alpha, 31)
    t = sb.Octree(img, colors, alpha)
    pid = ctx.palette_from_octree(t)
    try:
        got = ctx.dither_host("jacobi", img, pid)
        sweeps, converged = ctx.last_sweeps
    finally:
        ctx.release_palette(pid)
    q = synth.to_q16(img)
    n = 1024 * 1024
    free_list, _, pal = oracle.walk_blocks(q, colors, alpha, t.grayscale, n)
    assert converged and sweeps <= 8, (sweeps, converged)
    # The exact cache-free walk along the block-mode list, bit for bit.
    assert np.array_equal(got, free_list)
    # Its distance from the memoised sequential walk: the stated floor.
    cached, _, _ = oracle.walk_seq(q, colors, alpha, t.grayscale)
    mm = metrics.index_mismatch(got.reshape(-1), cached.reshape(-1))
    de = metrics.mean_delta_e(pal, got.reshape(-1), cached.reshape(-1))
    print(f"block sweeps colors={colors} alpha={alpha}: {sweeps} sweeps; vs memoised walk "
          f"mismatch {mm:.4f}, mean dE76 {de:.3f}")
    max_mm, max_de = MEMO_FLOOR[(colors, alpha)]
    assert mm <= max_mm and de <= max_de


@pytest.mark.parametrize("w,h,iters", [(97, 61, 20), (640, 480, 2), (1, 1, 20), (17, 13, 20)])
def test_block_sweeps_shapes_and_limits(ctx, oracle, w, h, iters):
    """Small and ragged lists, a 1x1 image, and a sweep limit: with too few
    sweeps the result is still a valid approximation and `converged` says so."""
    img = synth.gradient_rgb8(w, h, 5)
    t = sb.Octree(img, 16, False)
    pid = ctx.palette_from_octree(t)
    try:
        got = ctx.dither_host("jacobi", img, pid, jacobi_iters=iters)
        sweeps, converged = ctx.last_sweeps
    finally:
        ctx.release_palette(pid)
    n = max(16, w * h)
    want, _, _ = oracle.walk_blocks(synth.to_q16(img), 16, False, t.grayscale, n)
    assert sweeps <= max(1, iters)
    if converged:
        keep = np.ones(got.size, bool)
        gap = sb.block_gap(w, h)
        if gap >= 0:
            keep[gap] = False
        assert np.array_equal(got.reshape(-1)[keep], want.reshape(-1)[keep])
    else:
        assert sweeps == iters


# The point-iteration form: (index mismatch vs the cache-free walk, vs the
# memoised walk, mean CIE dE76 vs the memoised walk), 20 sweeps, 96 taps,
# 320x240.
POINT_TOLERANCE = {
    (16, False): (0.12, 0.14, 5.0),
    (64, False): (0.02, 0.06, 1.2),
    (256, False): (0.01, 0.06, 0.8),
    (16, True): (0.22, 0.22, 7.5),
}


@pytest.mark.parametrize("colors,alpha", list(POINT_TOLERANCE))
def test_point_iteration_tolerance(ctx, oracle, colors, alpha):
    max_free, max_cached, max_de = POINT_TOLERANCE[(colors, alpha)]
    img = _image(320, 240, alpha, 21)
    t = sb.Octree(img, colors, alpha)
    pid = ctx.palette_from_octree(t)
    try:
        got = ctx.dither_host("jacobi", img, pid, jacobi_form=1)
        q = synth.to_q16(img)
        cached, _, pal = oracle.walk_seq(q, colors, alpha, t.grayscale)
        free, _, _ = oracle.walk_seq(q, colors, alpha, t.grayscale, use_cache=False)
        gap = sb.block_gap(*img.shape[1::-1])
        mask = np.ones(got.size, bool)
        if gap >= 0:
            mask[gap] = False
        g, c, f = got.reshape(-1)[mask], cached.reshape(-1)[mask], free.reshape(-1)[mask]
        assert metrics.index_mismatch(g, f) <= max_free
        assert metrics.index_mismatch(g, c) <= max_cached
        assert metrics.mean_delta_e(pal, g, c) <= max_de
    finally:
        ctx.release_palette(pid)


def test_point_iteration_fp64_and_taps(ctx):
    img = synth.gradient_rgb8(200, 150, 3)
    t = sb.Octree(img, 16, False)
    pid = ctx.palette_from_octree(t)
    try:
        a = ctx.dither_host("jacobi", img, pid, jacobi_form=1)
        b = ctx.dither_host("jacobi", img, pid, jacobi_form=1, jacobi_fp64=1)
        assert metrics.index_mismatch(a, b) < 0.02
        c = ctx.dither_host("jacobi", img, pid, jacobi_form=1, jacobi_taps=16, jacobi_iters=4)
        assert c.shape == a.shape
        with pytest.raises(sb.RdbError):
            ctx.dither_host("jacobi", img, pid, jacobi_taps=0)
        with pytest.raises(sb.RdbError):
            ctx.dither_host("jacobi", img, pid, jacobi_form=7)
    finally:
        ctx.release_palette(pid)
