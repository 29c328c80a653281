"""Video frames through the blocks engine (rdb_dither_frames*): the decoder's
formats are widened in the gather and the encoder's formats written by the
scatter.  Byte-identical to the reference's host block walk with its fused
gather and output (RiemersmaBlocksCpu gather_raw / raw_out), compiled from
the reference's sources; 4:2:0 input, which the reference has on its CUDA
engine only, against the oracle's restatement of that gather."""
from __future__ import annotations

import numpy as np
import pytest

import stipple_b200 as sb
from stipple_b200 import synth

pytestmark = pytest.mark.gpu

GEOMS = [(64, 48), (37, 29), (2, 1), (1, 1), (256, 192), (130, 66)]
OUTS = [sb.RGBA16, sb.YUV444P8, sb.RGBAF32]


def _frames8(w, h, n, seed, alpha):
    fr = [synth.video_frame(w, h, seed, k) for k in range(n)]
    if alpha:
        a = synth.alpha_mask(w, h, seed)
        fr = [np.concatenate([f, a[:, :, None]], axis=2) for f in fr]
    return fr


def _decoder_frames(fmt, fr8, seed):
    """(raw (F, bytes) uint8, reference gather (layout, channels) or None)."""
    if fmt in (sb.RGB16, sb.RGBA16):
        raw = [synth.rgb16_frame(f, seed + k) for k, f in enumerate(fr8)]
        gather = (4, 3 if fmt == sb.RGB16 else 4)
    elif fmt == sb.YUV444P8:
        raw = [synth.yuv444_frame(f) for f in fr8]
        gather = (3, 0)
    elif fmt == sb.YUV420P8:
        raw = [synth.yuv420_frame(f) for f in fr8]
        gather = None
    elif fmt == sb.RGBAF32:
        raw = [synth.to_q16(f) for f in fr8]
        gather = (0, 0)
    else:  # RGB8 / RGBA8: the reader's widening is v * 257
        raw = list(fr8)
        gather = (0, 0)
    return np.stack([np.ascontiguousarray(r).reshape(-1).view(np.uint8) for r in raw]), gather


def _reference(reflib, oracle, tree_src, raw, fmt, gather, w, h, out_fmt, colors, assoc, block):
    """The reference's own bytes for the fused forms it has; the oracle's
    otherwise (RgbaF output is the non-fused walk, restated and pinned)."""
    if gather is not None and out_fmt != sb.RGBAF32:
        layout, ch = gather
        src = raw
        if layout == 0:
            src = np.stack([oracle.widen_frame(fmt, r, w, h) for r in raw])
        rc, msg, out = reflib.walk_blocks_raw(tree_src, src, layout, ch, w, h,
                                              out_fmt == sb.YUV444P8, colors, assoc, block)
        assert rc == 0, msg
        return out
    out, _ = oracle.walk_blocks_raw(tree_src, raw, fmt, w, h, out_fmt, colors, assoc, block)
    return out


def _palette(ctx, tree_src, colors, assoc):
    return ctx.palette_from_octree(sb.Octree(tree_src, colors, assoc))


@pytest.mark.parametrize("fmt", [sb.RGB16, sb.RGBA16, sb.YUV444P8, sb.RGBAF32, sb.RGB8, sb.RGBA8])
def test_frames_match_reference(ctx, reflib, oracle, fmt):
    alpha_in = fmt in (sb.RGBA16, sb.RGBAF32, sb.RGBA8)
    for k, (w, h) in enumerate(GEOMS):
        fr8 = _frames8(w, h, 3, 70 + k, alpha_in)
        raw, gather = _decoder_frames(fmt, fr8, 90 + k)
        tree_src = oracle.widen_frame(fmt, raw[0], w, h)
        for assoc in ([False, True] if alpha_in else [False]):
            colors = 64 if k % 2 else 256
            pid = _palette(ctx, tree_src, colors, assoc)
            try:
                for block in (32, 512):
                    for out_fmt in OUTS:
                        got = ctx.dither_frames_host(raw, fmt, w, h, pid, out_fmt, block=block)
                        want = _reference(reflib, oracle, tree_src, raw, fmt, gather, w, h,
                                          out_fmt, colors, assoc, block)
                        assert np.array_equal(got, want), (fmt, out_fmt, w, h, assoc, block)
            finally:
                ctx.release_palette(pid)


def test_frames_yuv420_match_oracle(ctx, oracle):
    for k, (w, h) in enumerate([(64, 48), (38, 30), (2, 2), (256, 192), (130, 66)]):
        fr8 = _frames8(w, h, 2, 40 + k, False)
        raw, _ = _decoder_frames(sb.YUV420P8, fr8, 0)
        tree_src = oracle.widen_frame(sb.YUV420P8, raw[0], w, h)
        pid = _palette(ctx, tree_src, 128, False)
        try:
            for out_fmt in OUTS:
                got = ctx.dither_frames_host(raw, sb.YUV420P8, w, h, pid, out_fmt, block=256)
                want, _ = oracle.walk_blocks_raw(tree_src, raw, sb.YUV420P8, w, h, out_fmt, 128,
                                                 False, 256)
                assert np.array_equal(got, want), (out_fmt, w, h)
        finally:
            ctx.release_palette(pid)


def test_frames_index_maps(ctx, oracle):
    """The index maps equal the oracle's block walk of each widened frame; the
    block list's gap is left unwritten (0) as in rdb_dither."""
    w, h = 256, 192
    fr8 = _frames8(w, h, 2, 5, False)
    raw, _ = _decoder_frames(sb.YUV444P8, fr8, 0)
    tree_src = oracle.widen_frame(sb.YUV444P8, raw[0], w, h)
    pid = _palette(ctx, tree_src, 256, False)
    try:
        _, idx = ctx.dither_frames_host(raw, sb.YUV444P8, w, h, pid, sb.YUV444P8, indices=True,
                                        block=64)
        _, want = oracle.walk_blocks_raw(tree_src, raw, sb.YUV444P8, w, h, sb.YUV444P8, 256,
                                         False, 64)
        assert np.array_equal(idx, want)
        gap = sb.block_gap(w, h)
        assert gap >= 0 and np.all(idx.reshape(2, -1)[:, gap] == 0)
    finally:
        ctx.release_palette(pid)


def test_frames_device_form_strided_and_in_place(ctx, oracle):
    """Device buffers with frame pitches wider than a frame, on a caller's
    stream; an RgbaF batch dithered in place equals the out-of-place result."""
    import torch
    w, h, nf = 130, 66, 3
    fr8 = _frames8(w, h, nf, 11, True)
    raw, _ = _decoder_frames(sb.RGBA16, fr8, 3)
    tree_src = oracle.widen_frame(sb.RGBA16, raw[0], w, h)
    pid = _palette(ctx, tree_src, 200, True)
    try:
        fb = sb.frame_bytes(sb.RGBA16, w, h)
        ob = sb.frame_bytes(sb.YUV444P8, w, h)
        dev = torch.device("cuda", 0)
        inp = torch.zeros((nf, fb + 64), dtype=torch.uint8, device=dev)
        inp[:, :fb] = torch.from_numpy(raw).to(dev)
        out = torch.full((nf, ob + 48), 7, dtype=torch.uint8, device=dev)
        s = torch.cuda.Stream(dev)
        ctx.dither_frames(inp.data_ptr(), sb.RGBA16, w, h, nf, pid, out.data_ptr(), sb.YUV444P8,
                          in_frame_bytes=fb + 64, out_frame_bytes=ob + 48, stream=s.cuda_stream,
                          block=128)
        ctx.synchronize(s.cuda_stream)
        got = out.cpu().numpy()
        want = ctx.dither_frames_host(raw, sb.RGBA16, w, h, pid, sb.YUV444P8, block=128)
        assert np.array_equal(got[:, :ob], want)
        assert np.all(got[:, ob:] == 7)  # the padding is not written

        q = np.stack([oracle.widen_frame(sb.RGBA16, r, w, h) for r in raw])
        buf = torch.from_numpy(q).to(dev).contiguous()
        ctx.dither_frames(buf.data_ptr(), sb.RGBAF32, w, h, nf, pid, buf.data_ptr(), sb.RGBAF32,
                          block=128)
        ctx.synchronize()
        want = ctx.dither_frames_host(q, sb.RGBAF32, w, h, pid, sb.RGBAF32, block=128)
        assert np.array_equal(buf.cpu().numpy().reshape(nf, -1).view(np.uint8), want)
    finally:
        ctx.release_palette(pid)


def test_frames_refusals(ctx, oracle):
    w, h = 33, 20
    raw, _ = _decoder_frames(sb.YUV444P8, _frames8(w, h, 1, 1, False), 0)
    pid = _palette(ctx, oracle.widen_frame(sb.YUV444P8, raw[0], w, h), 16, False)
    try:
        import torch
        # Room for either frame at either offset: the host refuses these
        # before anything is enqueued.
        buf = torch.zeros(16384, dtype=torch.uint8, device="cuda")
        with pytest.raises(sb.RdbError, match="even width and height"):
            ctx.dither_frames(buf.data_ptr(), sb.YUV420P8, w, h, 1, pid, buf.data_ptr() + 8192,
                              sb.YUV444P8)
        with pytest.raises(sb.RdbError, match="in place"):
            ctx.dither_frames(buf.data_ptr(), sb.YUV444P8, w, h, 1, pid, buf.data_ptr(),
                              sb.YUV444P8)
        with pytest.raises(sb.RdbError, match="output frame format"):
            ctx.dither_frames_host(raw, sb.YUV444P8, w, h, pid, sb.RGB8)
        with pytest.raises(sb.RdbError, match="at least 16"):
            ctx.dither_frames_host(raw, sb.YUV444P8, w, h, pid, sb.YUV444P8, block=8)
        with pytest.raises(sb.RdbError, match="unknown palette"):
            ctx.dither_frames_host(raw, sb.YUV444P8, w, h, pid + 1000, sb.YUV444P8)
    finally:
        ctx.release_palette(pid)


def test_frames_4k_yuv444_match_reference(ctx, reflib, oracle):
    """Two 3840x2160 planar 4:4:4 frames, 256 colours, rgba64 and 4:4:4 out."""
    w, h = 3840, 2160
    fr8 = [synth.video_frame(w, h, 2024, k) for k in range(2)]
    raw, _ = _decoder_frames(sb.YUV444P8, fr8, 0)
    tree_src = oracle.widen_frame(sb.YUV444P8, raw[0], w, h)
    pid = _palette(ctx, tree_src, 256, False)
    try:
        for out_fmt in (sb.YUV444P8, sb.RGBA16):
            got = ctx.dither_frames_host(raw, sb.YUV444P8, w, h, pid, out_fmt, block=512)
            rc, msg, want = reflib.walk_blocks_raw(tree_src, raw, 3, 0, w, h,
                                                   out_fmt == sb.YUV444P8, 256, False, 512)
            assert rc == 0, msg
            assert np.array_equal(got, want), out_fmt
    finally:
        ctx.release_palette(pid)
