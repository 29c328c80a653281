"""The device-assisted palette build (rdb_octree_build_device) against the
reference's ColorTree::Build (src/rd_octree.cpp:219-409): the colormap bit for
bit and the live tree node for node (structure, pixel counts, colour numbers)
-- the node array lists live nodes in another order than the host build, so
trees are compared by a walk from the root in child-id order.  Inputs: the
golden fixtures (the reference's own test images), greyscale (depth 8), alpha
association, RgbaF input, and seeded images across the served size range
(64..4096 per side) and colour counts 2..256."""
from __future__ import annotations

import numpy as np
import pytest

import golden
import stipple_b200 as sb
from stipple_b200 import synth

pytestmark = pytest.mark.gpu


def _live(child, cn, nu, fan):
    out = []
    stack = [(0, 0, 0)]
    while stack:
        node, level, ident = stack.pop()
        out.append((level, ident, int(nu[node]), int(cn[node]) if nu[node] else -1))
        for i in reversed(range(fan)):
            c = int(child[node, i])
            if c >= 0:
                stack.append((c, level + 1, i))
    return out


def _check(ctx, oracle, img, colors, alpha, gray, expect_device=True):
    import torch
    d = torch.from_numpy(np.ascontiguousarray(img)).cuda()
    lay = sb.layout_of(img)
    h, w = img.shape[:2]
    t, rows = ctx.octree_device(d.data_ptr(), lay, w, h, colors, alpha, gray)
    q = img if img.dtype == np.float32 else synth.to_q16(img)
    want = oracle.build_tree(q, colors, alpha, gray)
    assert np.array_equal(t.colormap(), want.palette), (w, h, colors, alpha)
    child, _, cn, nu = t.nodes()
    fan = 16 if alpha else 8
    assert _live(child, cn, nu, fan) == _live(want.child, want.color_number, want.number_unique, fan)
    if expect_device:
        assert rows > 0, "the device classified no rows"
    return rows


def test_golden_inputs(ctx, oracle):
    for name, rgbaf, recs in golden.cases():
        for r in recs:
            colors, assoc, gray = int(r["colors"]), bool(r["assoc"]), bool(r["gray"])
            _check(ctx, oracle, rgbaf, colors, assoc, gray, expect_device=False)


@pytest.mark.parametrize("w,h", [(64, 64), (97, 211), (640, 480), (1920, 1080), (4096, 1024)])
@pytest.mark.parametrize("colors", [2, 16, 256])
def test_sizes_and_colours(ctx, oracle, w, h, colors):
    _check(ctx, oracle, synth.gradient_rgb8(w, h, w + colors), colors, False, False)


@pytest.mark.parametrize("colors", [4, 64, 256])
def test_alpha(ctx, oracle, colors):
    _check(ctx, oracle, synth.gradient_rgba8(800, 600, colors), colors, True, False)


def test_greyscale_depth8(ctx, oracle):
    img = synth.gradient_rgb8(512, 384, 9)
    img[..., 1] = img[..., 0]
    img[..., 2] = img[..., 0]
    _check(ctx, oracle, img, 16, False, True)


def test_float_input(ctx, oracle):
    q = synth.to_q16(synth.gradient_rgb8(300, 200, 4))
    q[..., :3] += np.float32(0.25)  # fractional Q16 values
    _check(ctx, oracle, q, 64, False, False)


def test_flat_runs(ctx, oracle):
    """Long runs of equal pixels (weights above 1) and rows that repeat."""
    img = np.repeat(np.repeat(synth.gradient_rgb8(40, 30, 2), 8, axis=1), 4, axis=0)
    _check(ctx, oracle, img, 32, False, False)


def test_profiled_build_reports_its_parts(ctx, oracle):
    """With profiling on, the build's wall time by part: the host's first loop,
    the device classification and the host reduction each took some."""
    img = synth.gradient_rgb8(640, 480, 17)
    ctx.profile(True)
    try:
        _check(ctx, oracle, img, 64, False, False)
        parts = list(ctx.stats()["octree_ms"])
    finally:
        ctx.profile(False)
    assert parts[0] > 0 and parts[1] > 0 and parts[3] > 0, parts
