"""Block engine on the GPU: bit-exact against the reference's host block walk
(RiemersmaBlocksCpu), owner-map scatter and unvisited cell included."""
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


@pytest.mark.parametrize("name,rgbaf,recs", list(golden.cases()),
                         ids=lambda v: v if isinstance(v, str) else "")
def test_blocks_match_golden(ctx, oracle, name, rgbaf, recs):
    h, w = rgbaf.shape[:2]
    for r in recs:
        colors, assoc, gray = int(r["colors"]), bool(r["assoc"]), bool(r["gray"])
        tree = oracle.build_tree(rgbaf, colors, assoc, gray)
        pid = ctx.palette(tree.palette, tree.child, tree.color_number, tree.number_unique, assoc,
                          parent=tree.parent)
        try:
            for key in [k for k in r if k.startswith("blk")]:
                b = int(key[3:])
                idx, rgba = ctx.dither_host("blocks", rgbaf, pid, rgba=True, block=b)
                keep = np.ones(h * w, bool)
                keep[r[f"kept{b}"]] = False
                got = idx.reshape(-1)[keep]
                assert np.array_equal(_colours(r["pal"], got, assoc),
                                      _colours(r["pal"], r[key].reshape(-1)[keep], assoc)), (name, colors, b)
                # The unvisited cell keeps its source value in the RgbaF result.
                assert np.array_equal(rgba.reshape(-1, 4)[~keep], rgbaf.reshape(-1, 4)[~keep])
        finally:
            ctx.release_palette(pid)


@pytest.mark.parametrize("alpha", [False, True])
def test_blocks_match_oracle_seeded(ctx, oracle, alpha):
    for k, (w, h) in enumerate([(2, 1), (3, 5), (64, 64), (256, 192), (300, 170), (1024, 768)]):
        for colors in (4, 64, 256):
            img = synth.gradient_rgba8(w, h, 50 + k) if alpha else synth.gradient_rgb8(w, h, 50 + k)
            t = sb.Octree(img, colors, alpha)
            pid = ctx.palette_from_octree(t)
            try:
                for block in (16, 37, 256, 4096):
                    idx = ctx.dither_host("blocks", img, pid, block=block)
                    oidx, _, _ = oracle.walk_blocks(synth.to_q16(img), colors, alpha, t.grayscale, block)
                    gap = sb.block_gap(w, h)
                    if gap >= 0:
                        idx.reshape(-1)[gap] = oidx.reshape(-1)[gap] = 0
                    assert np.array_equal(idx, oidx), (w, h, colors, block)
            finally:
                ctx.release_palette(pid)


def test_blocks_one_by_one_is_untouched(ctx):
    img = np.array([[[10, 20, 30]]], np.uint8)
    t = sb.Octree(img, 16, False)
    pid = ctx.palette_from_octree(t)
    try:
        q = synth.to_q16(img)
        # BuildCurveIndex is empty at level 0: the pixel keeps its source value.
        _, rgba = ctx.dither_host("blocks", q, pid, rgba=True)
        assert np.array_equal(rgba, q)
        _, rgba = ctx.dither_host("blocks", img, pid, rgba=True)
        assert np.array_equal(rgba, q)
    finally:
        ctx.release_palette(pid)


def test_blocks_refusals(ctx):
    img = synth.gradient_rgb8(32, 32, 1)
    t = sb.Octree(img, 16, False)
    pid = ctx.palette_from_octree(t)
    try:
        with pytest.raises(sb.RdbError):
            ctx.dither_host("blocks", img, pid, block=15)
    finally:
        ctx.release_palette(pid)


def test_blocks_video_batch(ctx, oracle):
    """A batch of frames sharing one palette: per-frame equality with the oracle."""
    frames = [synth.video_frame(320, 180, 4, f) for f in range(6)]
    t = sb.Octree(frames[0], 256, False)
    pid = ctx.palette_from_octree(t)
    try:
        got = ctx.dither_host("blocks", frames, [pid] * len(frames), block=512)
        for f, img in enumerate(frames):
            # The palette comes from frame 0; the oracle walk rebuilds it from
            # each frame, so walk frame 0's tree over every frame instead.
            oidx = oracle_blocks_with_tree(oracle, frames[0], img, 256, 512)
            assert np.array_equal(got[f], oidx), f
    finally:
        ctx.release_palette(pid)


def oracle_blocks_with_tree(oracle, palette_src, img, colors, block):
    """Oracle block walk of `img` under the palette built from `palette_src`."""
    import ctypes as C
    raw = oracle.build_tree_raw(synth.to_q16(palette_src), colors, False, False)
    try:
        h, w = img.shape[:2]
        count = raw.color_count
        pal = np.ctypeslib.as_array(raw.colormap, shape=(count * 4,)).copy()
        out = synth.to_q16(img).reshape(-1).copy()
        idx = np.zeros(w * h, np.uint8)
        assert oracle.lib.orc_walk_blocks(C.byref(raw), pal, count, 0, 1.0, block, w, h, out, idx) == 0
        return idx.reshape(h, w)
    finally:
        oracle.lib.orc_tree_free(C.byref(raw))


@pytest.mark.parametrize("w,h,colors,block,alpha", [(256, 192, 64, 37, False), (100, 37, 16, 256, False),
                                                     (64, 48, 8, 16, True)])
def test_idx_bin_dump(ctx, oracle, tmp_path, w, h, colors, block, alpha):
    """rdb_context_dump_indices: the chosen index at every block-list position,
    list order, images in call order -- the reference's `.idx.bin`."""
    imgs = [(synth.gradient_rgba8 if alpha else synth.gradient_rgb8)(w, h, s) for s in (5, 6)]
    t = sb.Octree(imgs[0], colors, alpha)
    pid = ctx.palette_from_octree(t)
    prefix = str(tmp_path / "dump")
    ctx.dump_indices(prefix)
    try:
        ctx.dither_host("blocks", imgs, [pid, pid], block=block)
    finally:
        ctx.dump_indices(None)
        ctx.release_palette(pid)
    got = np.fromfile(prefix + ".idx.bin", np.uint8)
    # The oracle builds its tree from the image it walks: walk each image with
    # the first image's tree by building from the first and checking both
    # images' lists in order.
    want = []
    for img in imgs:
        want.append(oracle.block_chosen_with_tree(synth.to_q16(imgs[0]), synth.to_q16(img), colors,
                                                  alpha, t.grayscale, block))
    assert np.array_equal(got, np.concatenate(want))
