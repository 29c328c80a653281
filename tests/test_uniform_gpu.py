"""The uniform-key table: every key it marks uniform must give its colour for
every target inside the key's box under the reference lookup (descent +
ClosestColor), corners and edges of the box included."""
from __future__ import annotations

import numpy as np
import pytest

from stipple_b200 import synth

pytestmark = pytest.mark.gpu


def _key_of(q: np.ndarray) -> np.ndarray:
    """rd_types.h:141-153 for clamped float32 targets: top 6 bits of each byte."""
    q = q.astype(np.float32)
    b = np.minimum(255, (np.trunc(2.0 * q.astype(np.float64)).astype(np.int64) + 257) // 514)
    k = b >> 2
    return k[:, 0] | (k[:, 1] << 6) | (k[:, 2] << 12)


@pytest.mark.parametrize("colors,gray", [(256, False), (16, False), (64, False), (16, True)])
def test_uniform_keys_match_search(ctx, oracle, colors, gray):
    img = synth.gradient_rgb8(320, 240, 17)
    if gray:
        img = img[..., :1].repeat(3, axis=2).copy()
    q = synth.to_q16(img)
    tree = oracle.build_tree(q, colors, False, gray)
    pid = ctx.palette(tree.palette, tree.child, tree.color_number, tree.number_unique, False,
                      parent=tree.parent)
    try:
        table = ctx.uniform_table(pid)
    finally:
        ctx.release_palette(pid)
    uni = np.nonzero(table != 255)[0]
    assert len(uni) > (1 << 18) // 4, "suspiciously few uniform keys"
    rng = np.random.default_rng(colors)
    keys = rng.choice(uni, size=min(1500, len(uni)), replace=False)
    kc = np.stack([keys & 63, (keys >> 6) & 63, keys >> 12], axis=1).astype(np.float64)
    lo = np.maximum(0.0, 1028.0 * kc - 128.5)
    hi = np.minimum(65535.0, 1028.0 * kc + 899.5)
    pts = []
    for corner in range(8):  # the box's corners (upper bounds are exclusive: 0.01 inside)
        sel = np.array([(corner >> c) & 1 for c in range(3)], bool)
        p = np.where(sel, np.where(hi >= 65535.0, 65535.0, hi - 0.01), lo)
        pts.append(p)
    for _ in range(4):
        pts.append(lo + rng.random(lo.shape) * (hi - lo))
    pts = np.concatenate(pts).astype(np.float32)
    kk = np.tile(keys, 12)
    inside = _key_of(pts) == kk
    assert inside.mean() > 0.9
    pts, kk = pts[inside], kk[inside]
    targets = np.concatenate([pts.astype(np.float64), np.full((len(pts), 1), 65535.0)], axis=1)
    got = oracle.lookups(q, colors, False, gray, targets)
    assert np.array_equal(got, table[kk].astype(np.int32))


def _key4_of(q: np.ndarray) -> np.ndarray:
    q = q.astype(np.float32)
    b = np.minimum(255, (np.trunc(2.0 * q.astype(np.float64)).astype(np.int64) + 257) // 514)
    k = b >> 2
    return k[:, 0] | (k[:, 1] << 6) | (k[:, 2] << 12) | (k[:, 3] << 18)


@pytest.mark.parametrize("colors", [256, 16])
def test_alpha_uniform_keys_match_search(ctx, oracle, colors):
    """Alpha-associated palettes (2^24 keys): the search target is associated
    once more inside ClosestColor, so the table's box argument runs on the
    associated coordinates; every key it marks must give its colour at the
    corners of its 4-channel box and inside it."""
    h, w = 200, 160
    rgb = synth.gradient_rgb8(w, h, 23)
    yy, xx = np.mgrid[0:h, 0:w]
    a = np.clip(40 + 200 * xx / w + np.random.default_rng(3).normal(0, 12, (h, w)), 0, 255)
    img = np.concatenate([rgb, a.astype(np.uint8)[:, :, None]], axis=2)
    q = synth.to_q16(img)
    tree = oracle.build_tree(q, colors, True, False)
    pid = ctx.palette(tree.palette, tree.child, tree.color_number, tree.number_unique, True,
                      parent=tree.parent)
    try:
        table = ctx.uniform_table(pid, alpha=True)
    finally:
        ctx.release_palette(pid)
    assert not np.any(table == 254)  # every key classified
    uni = np.nonzero(table != 255)[0]
    assert len(uni) > (1 << 24) // 50, "suspiciously few uniform keys"
    rng = np.random.default_rng(colors)
    keys = rng.choice(uni, size=min(600, len(uni)), replace=False)
    kc = np.stack([keys & 63, (keys >> 6) & 63, (keys >> 12) & 63, keys >> 18], axis=1).astype(np.float64)
    lo = np.maximum(0.0, 1028.0 * kc - 128.5)
    hi = np.minimum(65535.0, 1028.0 * kc + 899.5)
    pts = []
    for corner in range(16):
        sel = np.array([(corner >> c) & 1 for c in range(4)], bool)
        pts.append(np.where(sel, np.where(hi >= 65535.0, 65535.0, hi - 0.01), lo))
    for _ in range(4):
        pts.append(lo + rng.random(lo.shape) * (hi - lo))
    pts = np.concatenate(pts).astype(np.float32)
    kk = np.tile(keys, 20)
    inside = _key4_of(pts) == kk
    assert inside.mean() > 0.9
    pts, kk = pts[inside], kk[inside]
    got = oracle.lookups(q, colors, True, False, pts.astype(np.float64))
    assert np.array_equal(got, table[kk].astype(np.int32))
