"""The oracle's fused-format block walk (widen -> walk -> narrow, oracle.c)
pinned to the reference: against the golden vectors the reference's own
RiemersmaBlocksCpu wrote with gather_raw / raw_out, and against that build
directly on seeded frames when it is present.  Plus the library's frame-size
rule (no GPU needed)."""
from __future__ import annotations

import numpy as np
import pytest

import golden
from stipple_b200 import synth


def _oracle_fused(oracle, c, out_fmt):
    w, h = int(c["w"]), int(c["h"])
    layout, ch = int(c["layout"]), int(c["channels"])
    fmt = {(4, 3): 6, (4, 4): 8, (3, 0): 444, (0, 0): 16}[(layout, ch)]
    out, _ = oracle.walk_blocks_raw(c["tree_src"], c["inp"], fmt, w, h, out_fmt,
                                    int(c["colors"]), bool(c["assoc"]), int(c["block"]))
    return out


def test_oracle_frames_match_golden(oracle):
    n = 0
    for c in golden.frames():
        assert np.array_equal(_oracle_fused(oracle, c, 444), c["out_yuv"])
        assert np.array_equal(_oracle_fused(oracle, c, 8), c["out_rgba64"])
        n += 1
    assert n == 7


@pytest.mark.parametrize("w,h", [(64, 48), (37, 29), (2, 1), (1, 1)])
def test_oracle_frames_match_reference(oracle, reflib, w, h):
    fr8 = [synth.video_frame(w, h, 9, k) for k in range(2)]
    a = synth.alpha_mask(w, h, 9)
    fr8a = [np.concatenate([f, a[:, :, None]], axis=2) for f in fr8]
    for ch in (3, 4):
        src = fr8a if ch == 4 else fr8
        raw = np.stack([synth.rgb16_frame(f, k).reshape(-1).view(np.uint8) for k, f in enumerate(src)])
        fmt = 8 if ch == 4 else 6
        tree = oracle.widen_frame(fmt, raw[0], w, h)
        for assoc in ((False, True) if ch == 4 else (False,)):
            for yuv in (False, True):
                rc, msg, want = reflib.walk_blocks_raw(tree, raw, 4, ch, w, h, yuv, 16, assoc, 32)
                assert rc == 0, msg
                got, _ = oracle.walk_blocks_raw(tree, raw, fmt, w, h, 444 if yuv else 8, 16,
                                                assoc, 32)
                assert np.array_equal(got, want), (ch, assoc, yuv)
    raw = np.stack([synth.yuv444_frame(f).reshape(-1) for f in fr8])
    tree = oracle.widen_frame(444, raw[0], w, h)
    for yuv in (False, True):
        rc, msg, want = reflib.walk_blocks_raw(tree, raw, 3, 0, w, h, yuv, 64, False, 16)
        assert rc == 0, msg
        got, _ = oracle.walk_blocks_raw(tree, raw, 444, w, h, 444 if yuv else 8, 64, False, 16)
        assert np.array_equal(got, want), yuv


def test_oracle_yuv420_even_sample_is_a_copy(oracle):
    """4:2:0 chroma at even (x, y) is the stored sample itself, so a frame whose
    chroma is constant over each 2x2 quad widens like its 4:4:4 form."""
    w, h = 16, 10
    p444 = synth.yuv444_frame(synth.video_frame(w, h, 3, 0))
    p444[1:] = np.repeat(np.repeat(p444[1:, ::2, ::2], 2, axis=1), 2, axis=2)
    f420 = np.concatenate([p444[0].reshape(-1), p444[1, ::2, ::2].reshape(-1),
                           p444[2, ::2, ::2].reshape(-1)])
    a = oracle.widen_frame(420, f420, w, h)
    b = oracle.widen_frame(444, p444.reshape(-1), w, h)
    even = np.zeros((h, w), bool)
    even[::2, ::2] = True
    assert np.array_equal(a[even], b[even])
    with pytest.raises(ValueError):
        oracle.widen_frame(420, np.zeros(15 * 10 * 3 // 2, np.uint8), 15, 10)


def test_frame_bytes(lib):
    import stipple_b200 as sb
    assert sb.frame_bytes(sb.RGBA16, 3840, 2160) == 3840 * 2160 * 8
    assert sb.frame_bytes(sb.RGB16, 5, 3) == 90
    assert sb.frame_bytes(sb.YUV444P8, 1920, 1080) == 1920 * 1080 * 3
    assert sb.frame_bytes(sb.YUV420P8, 1920, 1080) == 1920 * 1080 * 3 // 2
    assert sb.frame_bytes(sb.YUV420P8, 1919, 1080) == 0
    assert sb.frame_bytes(sb.RGBAF32, 2, 2) == 64
    assert sb.frame_bytes(99, 2, 2) == 0
