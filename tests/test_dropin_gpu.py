"""The reference-facing C++ layer on the GPU, driven the way rdither's callers
drive it (reference ColorTree::Build, RgbaF frames in place) and compared with
the reference's own CPU engines compiled from its sources: the walk and the
"riemersma-b200" registry entry bit for bit with RiemersmaWalkCpu, the block
engine bit for bit with RiemersmaBlocksCpu, every frame independent."""
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
