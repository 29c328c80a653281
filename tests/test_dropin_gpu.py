"""The reference-facing C++ layer on the GPU, driven the way rdither's callers
drive it (reference ColorTree::Build, RgbaF frames in place) and compared with
the reference's own CPU engines compiled from its sources: the walk and the
"riemersma-b200" registry entry bit for bit with RiemersmaWalkCpu, the block
engine bit for bit with RiemersmaBlocksCpu (its fused decoder / encoder
formats included), every frame independent."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import pyoracle
from stipple_b200 import synth

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (pyoracle.dropin_available() and pyoracle.ref_available()),
                                 reason="drop-in layer or reference build absent")]


@pytest.fixture(scope="module")
def dropin():
    return pyoracle.DropinLib()


@pytest.fixture(scope="module")
def ref():
    return pyoracle.RefLib()


def _frames(w, h, n, alpha, seed):
    mk = synth.gradient_rgba8 if alpha else synth.gradient_rgb8
    return np.stack([synth.to_q16(mk(w, h, seed + f)) for f in range(n)])


@pytest.mark.parametrize("w,h,colors,alpha", [(200, 150, 16, False), (320, 240, 256, False),
                                              (160, 120, 64, True), (1, 1, 2, False)])
def test_walk_matches_reference_cpu(dropin, ref, w, h, colors, alpha):
    frames = _frames(w, h, 2, alpha, 5)
    src = frames[0].copy()
    got = frames.copy()
    err, dev = dropin.run("walk", src, got, colors, assoc=alpha)
    assert err == "", err
    assert "sm_10" in dev
    for f in range(2):
        want = ref.walk_seq_frame(src, frames[f], colors, alpha, False)
        assert np.array_equal(got[f].view(np.uint32), want.view(np.uint32)), f


def test_walk_params_and_plugin(dropin, ref):
    frames = _frames(256, 192, 1, False, 9)
    src = frames[0].copy()
    for diff, cache in ((0.5, True), (1.0, False)):
        got = frames.copy()
        err, _ = dropin.run("walk", src, got, 32, diffusion=diff, use_cache=cache)
        assert err == "", err
        want, _ = ref.walk_seq(frames[0], 32, False, False, diffusion=diff, use_cache=cache)
        assert np.array_equal(got[0].view(np.uint32), want.view(np.uint32)), (diff, cache)
    got = frames.copy()
    err, _ = dropin.run("plugin", src, got, 32)
    assert err == "", err
    want, _ = ref.walk_seq(frames[0], 32, False, False)
    assert np.array_equal(got[0].view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("block,slot", [(256, 0), (16, 1), (4096, 0)])
def test_blocks_match_reference_cpu(dropin, ref, block, slot):
    frames = _frames(256, 192, 3, False, 11)
    src = frames[0].copy()
    got = frames.copy()
    err, _ = dropin.run("blocks", src, got, 64, block=block, slot=slot)
    assert err == "", err
    want = frames.copy()
    rc, msg = ref.walk_blocks_frames(src, want, 64, False, False, block)
    assert rc == 0, msg
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_approx_runs_and_refuses(dropin):
    frames = _frames(160, 120, 1, False, 3)
    src = frames[0].copy()
    got = frames.copy()
    err, _ = dropin.run("approx", src, got, 16, iterations=10, taps=64)
    assert err == "", err
    assert not np.array_equal(got, frames)
    assert dropin.lib.dropin_max_frames(3840, 2160, 0) >= 1


# RiemersmaBlocksCuda's fused forms (BlockOptions::upload_u16 / in_mode /
# in_channels and emit_u16 / emit_yuv444) against RiemersmaBlocksCpu's
# gather_raw / raw_out; 4:2:0 (which only the reference's CUDA engine reads)
# against the oracle's restatement.
_MODES = {  # name: (in_mode, in_channels, reference gather layout / channels)
    "rgba64": (0, 4, (4, 4)), "rgb48": (0, 3, (4, 3)), "yuv444": (1, 0, (3, 0)),
    "yuv444_prepass": (2, 0, (3, 0)), "yuv420": (3, 0, None), "rgbaf": (None, 0, (0, 0)),
}


def _fused_input(mode, w, h, nf, alpha, seed):
    fr8 = [synth.video_frame(w, h, seed, k) for k in range(nf)]
    if alpha:
        a = synth.alpha_mask(w, h, seed)
        fr8 = [np.concatenate([f, a[:, :, None]], axis=2) for f in fr8]
    if mode in ("rgba64", "rgb48"):
        ch = 4 if mode == "rgba64" else 3
        raw = [synth.rgb16_frame(f[:, :, :ch], seed + k) for k, f in enumerate(fr8)]
        return np.stack([r.reshape(-1).view(np.uint8) for r in raw]), (8 if ch == 4 else 6)
    if mode in ("yuv444", "yuv444_prepass"):
        return np.stack([synth.yuv444_frame(f).reshape(-1) for f in fr8]), 444
    if mode == "yuv420":
        return np.stack([synth.yuv420_frame(f) for f in fr8]), 420
    return np.stack([synth.to_q16(f).reshape(-1).view(np.uint8) for f in fr8]), 16


@pytest.mark.parametrize("mode", list(_MODES))
@pytest.mark.parametrize("emit", ["rgba64", "yuv444", "rgbaf"])
def test_blocks_fused_forms_match_reference_cpu(dropin, ref, oracle, mode, emit):
    if mode == "rgbaf" and emit == "rgbaf":
        pytest.skip("the plain form, covered above")
    in_mode, ch, gather = _MODES[mode]
    w, h, nf = 256, 192, 3
    alpha = mode in ("rgba64", "rgbaf")
    for assoc in ((False, True) if alpha else (False,)):
        raw, fmt = _fused_input(mode, w, h, nf, alpha, 31)
        src = oracle.widen_frame(fmt, raw[0], w, h)
        widened = np.stack([oracle.widen_frame(fmt, r, w, h) for r in raw])
        batch = widened.copy() if mode == "rgbaf" else None
        if emit == "rgbaf":
            batch = np.zeros_like(widened)
            out = None
        else:
            out = np.zeros((nf, w * h * (3 if emit == "yuv444" else 8)), np.uint8)
        err = dropin.blocks_fused(src, nf, 64, assoc=assoc, block=256, batch=batch,
                                  in_raw=None if mode == "rgbaf" else raw,
                                  in_mode=in_mode or 0, in_channels=ch or 4, out_raw=out,
                                  emit_yuv444=emit == "yuv444")
        assert err == "", err
        if emit == "rgbaf":
            # Upload only: the RgbaF result of the widened frames, in place.
            want = widened.copy()
            rc, msg = ref.walk_blocks_frames(src, want, 64, assoc, False, 256)
            assert rc == 0, msg
            assert np.array_equal(batch.view(np.uint32), want.view(np.uint32)), (mode, assoc)
            continue
        if gather is None:
            want, _ = oracle.walk_blocks_raw(src, raw, fmt, w, h, 444 if emit == "yuv444" else 8,
                                             64, assoc, 256)
        else:
            layout, gch = gather
            rin = widened if layout == 0 else raw
            rc, msg, want = ref.walk_blocks_raw(src, rin, layout, gch, w, h, emit == "yuv444",
                                                64, assoc, 256)
            assert rc == 0, msg
        assert np.array_equal(out, want), (mode, emit, assoc)
